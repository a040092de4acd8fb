/*
 * voxviz_b200.h - C ABI of the B200-native GigaVoxels sparse-octree ray caster.
 *
 * Everything a caller binds is declared here: plain C types, raw pointers and
 * sizes, int status codes, no exceptions and no torch types.  Every entry point
 * names the reference interface it replaces (paths are relative to the
 * apecoraro/VoxVizThesis project root).
 *
 * Conventions
 *  - Volume space is the reference's normalized space [0,1]^3, Z up
 *    (GigaVoxelsRenderer.cpp:1674-1690 maps the world box to it; the builders
 *    here put the volume box at [0,1]^3 so world == normalized space).
 *  - A node is two uint32 words, exactly GigaVoxelsOctTree::Node::GpuDataStruct
 *    (GigaVoxelsOctTree.h:72-80, setters GigaVoxelsOctTree.cpp:1309-1383):
 *      word0: bit31 brick resident, bit30 constant node,
 *             bits 29..20 / 19..10 / 9..0 child-block base x / y / z in the
 *             node-pool grid (0,0,0 = no children)
 *      word1: constant node: RGBA8 r | g<<8 | b<<16 | a<<24
 *             otherwise:     brick pointer x<<20 | y<<10 | z (texel coords in
 *                            the brick-pool grid, already offset by the border)
 *  - Node-pool words passed across this ABI are in the reference texture order
 *    of OctTreeNodePool::create3DTexture (GigaVoxelsOctTree NodePool.cpp:90-223):
 *    a dim_x * dim_y * dim_z grid, x fastest, 2 words per node.
 *  - Bricks are 8^3 voxels stored with a 1-voxel border (10^3 texels), x
 *    fastest.  A brick-pool slot s = (sz*slots_y + sy)*slots_x + sx holds the
 *    texels of grid region [10*sx, 10*sx+10) x ... of the reference 3D texture
 *    (GigaVoxelsBrickPool.cpp:75-101), stored contiguously (brick-linear).
 *  - Functions that take a `vv_ctx` run on that context's CUDA device and
 *    stream.  Calls on one context must be externally serialised.
 */
#ifndef VOXVIZ_B200_H
#define VOXVIZ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VV_ABI_VERSION 1

/* Status codes (GigaVoxelsBrickPool.cpp:148-150 and GigaVoxelsReader.cpp:106-221
 * report failure as bool + std::cerr; here every call returns one of these). */
typedef enum vv_status {
    VV_OK = 0,
    VV_ERR_ARG = 1,      /* invalid argument or size                        */
    VV_ERR_OOM = 2,      /* device or host allocation failed                */
    VV_ERR_CUDA = 3,     /* CUDA runtime error                              */
    VV_ERR_TIMEOUT = 4,  /* a bounded device wait or loop ran out           */
    VV_ERR_BOUNDS = 5,   /* a device-side index check failed                */
    VV_ERR_STATE = 6,    /* call out of order (e.g. render before upload)   */
    VV_ERR_NODEV = 7,    /* no CUDA device / extension not usable           */
    VV_ERR_IO = 8        /* a file is missing, unreadable or malformed      */
} vv_status;

/* Brick-pool texel formats. RGBA8 is GL_RGBA8 (GigaVoxelsBrickPool.cpp:45);
 * the float formats hold the same normalized [0,1] values. */
typedef enum vv_fmt {
    VV_FMT_RGBA8 = 0,   /* 4 x uint8, unorm                              */
    VV_FMT_FP16 = 1,    /* 4 x IEEE binary16                             */
    VV_FMT_BF16 = 2,    /* 4 x bfloat16                                  */
    VV_FMT_FP32 = 3,    /* 4 x float                                     */
    /* S3TC block-compressed pools (GL_COMPRESSED_RGBA_S3TC_DXT5 colour and
     * GL_COMPRESSED_RGB_S3TC_DXT1 gradient textures of the reference,
     * GigaVoxelsRenderer.cpp:235-258): each brick's 10 z slices of 10x10
     * texels padded to 12x12 as 4x4 blocks, 90 blocks per slot, block
     * (z*9 + (y/4)*3 + x/4) of the slot, texel (y%4)*4 + x%4 of the block.
     * Decoded to RGBA8 values, then filtered like RGBA8.  The expansion and
     * interpolation rounding S3TC leaves open are fixed (voxviz_b200/csrc/
     * dxt.h).  DXT5 for brick pools (1440 bytes per slot), DXT1 for
     * gradient pools (720 bytes per slot, unsigned gradients). */
    VV_FMT_DXT5 = 4,
    VV_FMT_DXT1 = 5
} vv_fmt;

#define VV_BRICK_DIM 8          /* interior voxels per axis               */
#define VV_BRICK_STORED 10      /* stored texels per axis (1-voxel border) */
#define VV_BRICK_TEXELS 1000    /* texels per stored brick                */
#define VV_USAGE_SLOTS 12       /* node-usage entries per pixel (3 x RGBA32UI) */

/* Per-draw uniforms.  The first block is exactly the set of uniforms read by
 * VoxViz/Shaders/GigaVoxelsNoLighting.frag:3-26, derived on the host as
 * GigaVoxelsRenderer::drawVolume does (GigaVoxelsRenderer.cpp:1630-1816).
 * The second block replaces rasterisation of the volume box
 * (GigaVoxels.vert:11-19) and of the near-plane quad (NearPlaneQuad.vert:11-20):
 * pixel (px,py) (origin bottom-left, as gl_FragCoord) looks along
 * d = near_origin + (px+0.5)*near_dx + (py+0.5)*near_dy, the vector from the
 * camera to the pixel's near-plane point (camera-relative, so that small near
 * distances keep full float precision).  A camera outside the volume box
 * starts the ray at the box entry camera + t*d; a camera inside starts it at
 * the near-plane point camera + d. */
typedef struct vv_uniforms {
    float ray_step_size;           /* RayStepSize                          */
    float brick_step_vector[3];    /* BrickStepVector                      */
    float camera_position[3];      /* CameraPosition (normalized space)    */
    float camera_up[3];            /* CameraUp (unit, world)               */
    float camera_left[3];          /* CameraLeft (unit, world)             */
    float vol_extent_min[3];       /* VolExtentMin                         */
    float vol_extent_max[3];       /* VolExtentMax                         */
    float brick_dimension[3];      /* BrickDimension                       */
    float root_voxel_half_size;    /* RootVoxelHalfSize                    */
    float brick_pool_dimension[3]; /* BrickPoolDimension (texels)          */
    float pixel_size;              /* PixelSize                            */
    float lod_scalar;              /* LodScalar                            */
    float alpha_stop;              /* early-termination alpha (the shader's
                                      literal 0.995f; a parameter here)    */
    int32_t oct_tree_depth_minus_one; /* OctTreeDepthMinusOne             */
    int32_t max_nodes_to_push;     /* MaxNodesToPushThisFrame              */
    int32_t root_node_is_constant; /* RootNodeIsConstant                   */
    int32_t jitter_tex_size;       /* JitterTexSize                        */
    /* ray generation */
    int32_t width;
    int32_t height;
    int32_t camera_inside;         /* 1: rays start on the near plane      */
    int32_t max_segments;          /* loop bound per ray (0 = derived)     */
    float near_origin[3];
    float near_dx[3];
    float near_dy[3];
    /* Lighting: GigaVoxels.frag with ComputeLighting (:16, :27-28, shading
     * :293-312, LookupGradient :314-325, TraverseBrick :337, :370-384).
     * Off (0) in every benchmark configuration, which then follows
     * GigaVoxelsNoLighting.frag.  On needs a gradient pool
     * (vv_gradpool_create) and is supported by vv_render. */
    float light_position[3];       /* LightPosition, normalized volume space */
    int32_t compute_lighting;      /* ComputeLighting                        */
    int32_t gradients_unsigned;    /* GradientsAreUnsigned: texel*2 - 1      */
} vv_uniforms;

/* One node-word update (OctTreeNodePool::update3DTexture,
 * GigaVoxelsOctTreeNodePool.cpp:256-288). */
typedef struct vv_node_patch {
    uint32_t x, y, z;      /* node-pool grid position */
    uint32_t word0, word1;
} vv_node_patch;

/* Outputs of one draw.  Pointers are DEVICE pointers on the context's device
 * (NULL = not wanted; the context then uses internal scratch where a later
 * pass needs the data). */
typedef struct vv_frame_out {
    float* color;             /* [H][W][4] FragColor (before blending)        */
    uint32_t* usage;          /* [H][W][12] NodeUsageList[3] (GigaVoxels*.frag) */
    uint32_t* mask;           /* [H][W] selection mask (GenerateSelectionMask.frag) */
    uint32_t* requests;       /* [request_cap][4] CompressNodeUsageList output */
    uint32_t* request_count;  /* [1] active-pixel count (histopyramid top), uncapped */
    int32_t request_cap;      /* max compacted entries written (reference: 32768) */
    int32_t compress_max_push;/* CompressNodeUsageList MaxNodesToPushThisFrame  */
    int32_t passes;           /* VV_PASS_* bit set: which passes to run        */
} vv_frame_out;

#define VV_PASS_RAYCAST 1
#define VV_PASS_SELECT 2
#define VV_PASS_COMPACT 4
#define VV_PASS_ALL 7
/* With VV_PASS_RAYCAST: colour as RGBA8 unorm, round(clamp(c, 0, 1) * 255)
 * per channel (r in the low byte), into `color` read as uint32_t[H][W]:
 * 4 bytes per pixel instead of 16 (the display format of the frame). */
#define VV_PASS_COLOR_RGBA8 8

typedef struct vv_ctx vv_ctx;

typedef struct vv_params {
    int32_t device;       /* CUDA device ordinal */
    int32_t flags;        /* reserved, 0 */
    int64_t reserved[4];
} vv_params;

/* ---- context ---------------------------------------------------------- */

/* Replaces the GL context + BrickPool singleton set-up of
 * GigaVoxelsRenderer::init (GigaVoxelsRenderer.cpp:341-607). */
int vv_ctx_create(const vv_params* params, vv_ctx** out);
int vv_ctx_destroy(vv_ctx* ctx);
/* Last error message of this context ("" if none); valid until the next call. */
const char* vv_last_error(const vv_ctx* ctx);
const char* vv_status_string(int status);
/* Use this CUDA stream (cudaStream_t) for every later call; NULL = default. */
int vv_ctx_set_stream(vv_ctx* ctx, void* cuda_stream);
int vv_ctx_synchronize(vv_ctx* ctx);
/* Sticky device status word (VV_OK or the first device-side error code). */
int vv_ctx_device_status(vv_ctx* ctx, int32_t* status, int32_t clear);
int vv_abi_version(void);

/* ---- node pool ---------------------------------------------------------- */

/* Upload a whole node pool for octree slot `tree` (0..VV_MAX_TREES-1) from host
 * words in reference texture order.  Replaces OctTreeNodePool::create3DTexture
 * (GigaVoxelsOctTreeNodePool.cpp:90-223). dim_x/dim_y/dim_z must be even. */
#define VV_MAX_TREES 8
int vv_nodepool_upload(vv_ctx* ctx, int32_t tree, const uint32_t* words,
                       int32_t dim_x, int32_t dim_y, int32_t dim_z);
/* Apply n host-side patches.  Replaces OctTreeNodePool::update
 * (GigaVoxelsOctTreeNodePool.cpp:230-288). */
int vv_nodepool_patch(vv_ctx* ctx, int32_t tree, const vv_node_patch* patches,
                      int32_t n);
/* Read the node pool back in reference texture order (for checking). */
int vv_nodepool_download(vv_ctx* ctx, int32_t tree, uint32_t* words);
/* Grid dimensions of octree slot `tree` (0,0,0 if none was uploaded). */
int vv_nodepool_info(const vv_ctx* ctx, int32_t tree, int32_t dims[3]);

/* ---- brick pool ----------------------------------------------------------- */

/* Create the brick pool: slots_x*slots_y*slots_z slots of 10^3 texels in
 * `fmt`.  Replaces BrickPool::init / initSpecial (GigaVoxelsBrickPool.cpp:55-251).
 * slots_* * 10 must be <= 1023 (10-bit brick pointers). */
int vv_brickpool_create(vv_ctx* ctx, int32_t slots_x, int32_t slots_y,
                        int32_t slots_z, int32_t fmt);
/* Copy n bricks from host memory into the given slots.  `texels` holds n
 * consecutive bricks of 1000 texels in the pool's format.  Replaces the PBO
 * staging + glTexSubImage3D of BrickPool::uploadBrick / uploadPBOToTextures
 * (GigaVoxelsBrickPool.cpp:451-559,729-813). */
int vv_upload_bricks(vv_ctx* ctx, const uint32_t* slots, int32_t n,
                     const void* texels);
/* Same with device-resident brick data (`texels_dev`, `slots_dev` device ptrs). */
int vv_upload_bricks_device(vv_ctx* ctx, const uint32_t* slots_dev, int32_t n,
                            const void* texels_dev);
/* The gradient texture of the brick pool (BrickPool::getGradientTextureID,
 * GigaVoxelsBrickPool.cpp:820): the same slots, one gradient per texel, as
 * VV_FMT_FP32 (x, y, z, unused: the reference's Vec3f gradients) or
 * VV_FMT_RGBA8 (components stored as unsigned bytes; sampled /255 and, with
 * gradients_unsigned, mapped back by *2-1).  Create after the brick pool. */
int vv_gradpool_create(vv_ctx* ctx, int32_t fmt);
int vv_upload_gradients(vv_ctx* ctx, const uint32_t* slots, int32_t n, const void* texels);
int vv_gradpool_download(vv_ctx* ctx, void* texels);
/* Read the whole pool back (slot-major, brick-linear) into host memory. */
int vv_brickpool_download(vv_ctx* ctx, void* texels);
/* Slots per axis and format of the brick pool (0 slots if none exists). */
int vv_brickpool_info(const vv_ctx* ctx, int32_t slots[3], int32_t* fmt);
/* Device address of the pool texels (for callers that manage data on device).
 * After writing pool texels through it, call vv_brickpool_update_cell_masks. */
int vv_brickpool_device_ptr(vv_ctx* ctx, void** ptr, size_t* bytes);
/* Empty-cell masks (no counterpart in the reference: an acceleration of the
 * ray cast that leaves every result unchanged).  Per slot, bit
 * (z*9 + y)*9 + x of 32 uint32 words is set when the eight texels of the
 * 2x2x2 cell whose first texel is (x,y,z), x,y,z in [0,8], are zero in every
 * bit; a sample whose taps are such a cell is exactly zero, so the ray cast
 * takes the zero without reading texels.  The library keeps the masks for
 * pools it writes (creation, vv_upload_bricks*, the renderer's production);
 * vv_brickpool_attach leaves them invalid (no skipping) until
 * vv_brickpool_update_cell_masks rebuilds them from the pool's contents,
 * which is also the call to make after writing texels through
 * vv_brickpool_device_ptr or an attached buffer.  Download: slots*32 words,
 * VV_ERR_STATE while the masks are invalid. */
int vv_brickpool_update_cell_masks(vv_ctx* ctx);
int vv_brickpool_download_cell_masks(vv_ctx* ctx, uint32_t* words);

/* The 2D jitter texture (GLUtils::Create2DJitterTexture, GLUtils.cpp:455-497):
 * size*size uint8 values in [1,255], row-major. */
int vv_set_jitter(vv_ctx* ctx, const uint8_t* table, int32_t size);

/* ---- the hot path --------------------------------------------------------- */

/* One draw of octree `tree`: the ray cast of GigaVoxelsNoLighting.frag
 * (main :490-751), then GenerateSelectionMask.frag, ComputeActiveTexels.frag
 * + GenerateHistoPyramid.frag and CompressNodeUsageList.frag, as run by
 * GigaVoxelsRenderer::drawVolume / generateNodeUsageSelectionMask /
 * generateSelectionMaskHistoPyramid / compressNodeUsageList
 * (GigaVoxelsRenderer.cpp:1584-2135).  Asynchronous on the context stream. */
int vv_render(vv_ctx* ctx, int32_t tree, const vv_uniforms* u,
              const vv_frame_out* out);

/* Kernel timing: with profiling on, vv_render records CUDA events around the
 * ray cast and around the selection/compaction passes on the context stream
 * (the reference kept QElapsedTimer pass timers, GigaVoxelsRenderer.cpp:858-903).
 * vv_ctx_last_times waits for the last draw and returns its two durations. */
int vv_ctx_set_profiling(vv_ctx* ctx, int32_t on);
/* How vv_render's ray cast (unlit, colour and usage lists) is launched; the
 * results are the same.  VV_RAYCAST_TILES (default): one thread per pixel,
 * 16x8-pixel CTAs.  VV_RAYCAST_REFILL: a persistent grid whose warps take
 * 8x4-pixel tiles from a queue and run their rays one leaf segment at a
 * time, a lane whose ray has ended taking the next pixel (ballot + popc)
 * instead of idling until the warp's last ray ends.  VV_RAYCAST_STAGED
 * (RGBA8 pools only, else VV_ERR_ARG): the tiles launch, each warp copying
 * the brick slot that most of its lanes enter together into shared memory
 * (one cp.async.bulk of 4000 bytes) and those lanes sampling it there.  No
 * reference counterpart (one fragment per pixel in GL, bricks sampled
 * through the texture cache). */
#define VV_RAYCAST_TILES 0
#define VV_RAYCAST_REFILL 1
#define VV_RAYCAST_STAGED 2
int vv_ctx_set_raycast_mode(vv_ctx* ctx, int32_t mode);
/* How vv_render's selection + histopyramid + compaction are launched; the
 * results are the same.  VV_COMPACT_FUSED (default): three launches (the
 * selection and the pyramid's lowest five levels per 32x32-pixel node, the
 * levels above in one CTA, then the offsets down and the compaction), for
 * frames with at least 7 pyramid levels and at most 16384 level-5 nodes,
 * else the per-level form.  VV_COMPACT_PER_LEVEL: one launch per pyramid
 * level each way (GenerateHistoPyramid.frag's passes). */
#define VV_COMPACT_FUSED 0
#define VV_COMPACT_PER_LEVEL 1
int vv_ctx_set_compaction(vv_ctx* ctx, int32_t mode);
int vv_ctx_last_times(vv_ctx* ctx, float* raycast_ms, float* compact_ms);
/* Footprint of one draw: the number of distinct node-pool entries and
 * brick-pool slots the ray cast of `u` reads (a counting variant of the same
 * kernel; used for the algorithmic bytes of the roofline). */
int vv_measure_footprint(vv_ctx* ctx, int32_t tree, const vv_uniforms* u,
                         int64_t* nodes, int64_t* bricks);
/* The same for n draws of one batch: the distinct entries and slots of the
 * union of their reads (no reference counterpart: the roofline of a batched
 * launch). */
int vv_measure_footprint_views(vv_ctx* ctx, int32_t tree, const vv_uniforms* us, int32_t n,
                               int64_t* nodes, int64_t* bricks);

/* ---- differentiable ray cast --------------------------------------------- */

/* No counterpart in the reference: the adjoint of the ray cast with respect
 * to the brick texels.  vv_render_forward_ckpt runs the ray cast of vv_render
 * (colour only, identical values) and stores per-ray checkpoints (at a leaf
 * segment start every >= 32 composited samples, at most `per_ray` per ray)
 * into `ckpt`, a device buffer of vv_ckpt_bytes(width, height, per_ray)
 * bytes.  vv_backward then ADDS dL/d(texel) to `grad_texels` (device, one
 * float4 per pool texel, slot-major like the pool) given dL/d(colour)
 * (`dl_dcolor`, device, float4 per pixel) for the same uniforms and pools.
 * The gradient is with respect to the normalized texel value (v/255 for
 * RGBA8); the forward's control flow is held fixed. */
size_t vv_ckpt_bytes(int32_t width, int32_t height, int32_t per_ray);
int vv_render_forward_ckpt(vv_ctx* ctx, int32_t tree, const vv_uniforms* u, float* color,
                           void* ckpt, int32_t per_ray);
int vv_backward(vv_ctx* ctx, int32_t tree, const vv_uniforms* u, const float* dl_dcolor,
                const void* ckpt, int32_t per_ray, float* grad_texels);
/* Where vv_backward_ex adds the gradient.  `grad` holds 1000 texels per row,
 * 4 floats per texel, or 4 doubles with VV_GRAD_F64 (a binary64 reduction of
 * the per-sample contributions, for gradient checks).  With slot_map NULL
 * row = brick-pool slot (the dense layout of vv_backward).  With a slot map
 * (device, one int32 per pool slot, set to -1 by the caller before the
 * first call) the gradient is sparse: the first sample that reaches a slot
 * claims the next row (counter `rows_used`, device int32, zeroed by the
 * caller) and writes it into the map, so only touched slots take rows; the
 * caller zeroes the first `rows_cap` rows.  Running out of rows sets
 * VV_ERR_OOM in the device status (vv_ctx_device_status) and drops the
 * contributions that found no row.  Row order depends on timing; the map
 * tells which slot each row holds. */
#define VV_GRAD_F64 1
/* Lanes of a warp whose samples lie in the same brick cell (the same 8
 * texels) are summed with __match_any_sync and shuffles first, one atomic
 * per texel and cell group. */
#define VV_GRAD_WARP_SUM 2
/* Spread the atomics of a binary32 gradient (not with VV_GRAD_F64, else
 * VV_ERR_ARG) over VV_GRAD_SPREAD_COPIES copies of the rows: the four warps
 * of a CTA add to different copies (fewer concurrent atomics on one
 * address; eight copies would also separate neighbouring CTAs, for 1-3 %
 * on the paged frames at twice the memory).
 * The extra copies live in context memory ((copies - 1) * rows * 16000
 * bytes, rows = rows_cap with a slot map, else the pool's slots; kept
 * between calls) and are added into `grad` on the stream after the adjoint
 * (the rows in use with a slot map, every slot without).  Same gradient up
 * to the order of the float additions.  With VV_GRAD_SPREAD_KEEP as well
 * the sums stay in the copies; the next call with VV_GRAD_SPREAD and
 * without KEEP adds them into its `grad` - the calls in between must use
 * the same `grad`, slot map and row count (e.g. the views of one step). */
#define VV_GRAD_SPREAD 4
#define VV_GRAD_SPREAD_KEEP 8
#define VV_GRAD_SPREAD_COPIES 4
typedef struct vv_grad_desc {
    void* grad;
    int32_t flags;
    int32_t rows_cap;
    int32_t* slot_map;
    int32_t* rows_used;
} vv_grad_desc;
int vv_backward_ex(vv_ctx* ctx, int32_t tree, const vv_uniforms* u, const float* dl_dcolor,
                   const void* ckpt, int32_t per_ray, const vv_grad_desc* g);
/* Use caller-owned device memory (e.g. a torch tensor) as the brick pool:
 * slots_x*slots_y*slots_z*1000 texels of `fmt` at `texels`; the context does
 * not free it.  Replaces vv_brickpool_create for differentiable use. */
int vv_brickpool_attach(vv_ctx* ctx, void* texels, int32_t slots_x, int32_t slots_y,
                        int32_t slots_z, int32_t fmt);

/* ---- batched persistent ray cast ----------------------------------------- */

/* No counterpart in the reference (one drawVolume per octree per frame,
 * GigaVoxelsRenderer.cpp:1584-1935): many views of many octrees in ONE
 * launch.  A persistent grid pulls tile_w x tile_h pixel tiles of all views
 * from a device work queue; each pixel runs exactly the vv_render ray cast
 * of its view (colour and usage lists bit-identical to a per-view
 * vv_render with VV_PASS_RAYCAST).  Every view names the context holding
 * its octree's node pool (`tree`) and brick pool; all contexts must be on
 * the launching context's device and share one brick format.  The launch
 * runs on `ctx`'s stream and uses its scratch; the selection and
 * compaction passes of a view run afterwards through vv_render with
 * passes = VV_PASS_SELECT | VV_PASS_COMPACT on the same usage buffer. */
typedef struct vv_batch_view {
    vv_ctx* ctx;            /* context owning this view's pools           */
    int32_t tree;           /* node pool index in that context            */
    int32_t pad;
    vv_uniforms u;          /* the view's uniforms (as for vv_render)     */
    float* color;           /* device, 4 floats per pixel, or NULL: the
                               batched launch always writes float4 colour
                               (no RGBA8 form, unlike VV_PASS_COLOR_RGBA8) */
    uint32_t* usage;        /* device, 12 words per pixel, or NULL        */
} vv_batch_view;

typedef struct vv_batch_config {
    int32_t tile_w, tile_h;  /* pixel tile of one CTA: 8x8, 16x8, 16x16, 32x8 */
    int32_t steps;           /* march samples per loop trip: 1, 2 or 4      */
    int32_t ctas_per_sm;     /* resident CTAs per SM; 0 = occupancy limit   */
} vv_batch_config;

/* The compiled (tile_w, tile_h, steps) variants; returns their count and
 * writes up to `cap` of them. */
int32_t vv_batch_variants(vv_batch_config* out, int32_t cap);
int vv_render_batch(vv_ctx* ctx, const vv_batch_view* views, int32_t n, const vv_batch_config* cfg);
/* Times every compiled variant on this batch (one untimed launch, then
 * `reps` timed launches each, CUDA events on ctx's stream) and returns the
 * fastest in `best`.  `ms` (may be NULL) receives the mean launch time of
 * each variant in vv_batch_variants order.  The views' outputs hold the
 * last launch's results. */
int vv_batch_autotune(vv_ctx* ctx, const vv_batch_view* views, int32_t n, int32_t reps,
                      vv_batch_config* best, float* ms);

/* ---- page-request compaction without allocation ------------------------- */

/* This entry point has no counterpart in the reference.  It is for callers
 * that cannot call cudaMalloc: code that runs inside an allocator or a
 * memory-pool callback, a real-time render thread that must not block on the
 * driver's allocator, or a process whose device memory is owned by a
 * framework that forbids side allocations.  It needs no vv_ctx.
 *
 * Given a frame's node-usage lists (`usage`, width*height*12 words on the
 * device, as vv_render writes them) it writes the selection mask (`mask`,
 * width*height words), the compacted page requests (`requests`,
 * request_cap*4 words) and the active-pixel count (`request_count`, 1 word,
 * may be NULL) on `cuda_stream` - the same results as vv_render with
 * VV_PASS_SELECT | VV_PASS_COMPACT.  Inputs and outputs are the caller's; the
 * histopyramid lives in a 16 MiB file-scope device array that every GPU
 * loading the library holds until exit, so width*height may not exceed
 * VV_NOALLOC_MAX_PIXELS (2^21, enough for 1920x1080); larger frames return
 * VV_ERR_ARG.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress, with that device current); make that first
 * call before any stream capture.  That first call may also be the one that
 * loads the library's device code on that device (CUDA loads modules
 * lazily by default), which can allocate device memory and block; make it
 * once at start-up, outside the code that must not allocate.  The address
 * is kept for the life of the process: after cudaDeviceReset (or anything
 * else that destroys the device's primary context) the kept address is
 * stale, so do not call this entry point again in that process.  All calls share the one array: calls that
 * overlap on the GPU (different streams, or different host threads on the
 * same device) race and must be serialised by the caller.  It calls no
 * cudaMalloc, cudaFree or allocating library routine.  Errors: VV_ERR_ARG,
 * VV_ERR_CUDA; the message is in vv_last_error(NULL). */
#define VV_NOALLOC_MAX_PIXELS (1 << 21)
int vv_compact_requests_noalloc(const uint32_t* usage, uint32_t* mask, int32_t width,
                                int32_t height, uint32_t* requests, uint32_t* request_count,
                                int32_t request_cap, int32_t compress_max_push,
                                void* cuda_stream);

/* ---- host data model: terrain octree (GigaVoxelsOctTree) ----------------- */

typedef struct vv_octree vv_octree;

/* Synthetic terrain: seeded 2D fBm value-noise heightfield voxelised into a
 * (8 << depth)^3 volume; colour by 8 equal height bands. */
typedef struct vv_terrain_desc {
    uint32_t seed;
    int32_t depth;             /* leaf level L (OctTreeDepthMinusOne) */
    int32_t octaves;           /* 4 */
    float lacunarity;          /* 2.0 */
    float gain;                /* 0.5 */
    int32_t base_cells;        /* lattice cells across the volume at octave 0 */
    int32_t collapse_constant; /* 1: constant nodes are leaves (.gvx trees);
                                  0: full tree as GigaVoxelsOctTree::build */
    int32_t threads;           /* host threads for the build (0 = all) */
} vv_terrain_desc;

typedef struct vv_octree_info {
    int32_t depth;             /* L */
    int32_t volume_dim;        /* 8 << L */
    int64_t node_count;        /* allocated nodes (8 per block) */
    int32_t pool_dim[3];       /* node-pool grid */
    int64_t nonconst_count;    /* non-constant nodes (bricks that exist) */
    int32_t root_is_constant;
    uint32_t root_word0, root_word1;
} vv_octree_info;

/* GigaVoxelsOctTree::build (GigaVoxelsOctTree.cpp:1656-1701) for the terrain. */
int vv_octree_build_terrain(const vv_terrain_desc* desc, vv_octree** out);
/* The same tree built on CUDA device `device`: the heightfield, the 2x2x2
 * box-filter mip pyramid with round-half-up (GenerateMipMap /
 * GetBoxFilterAverage, GigaVoxelsOctTree.cpp:809-960; the voxelizer's
 * ComputeVoxelMipMap8, VoxelizerKernels.cu:1520) and the node
 * classification with the border rule (Node::computeNodeType, :1490-1609;
 * ComputeOctTreeNodeType, VoxelizerKernels.cu:2216) run as kernels; the host
 * numbers the blocks and keeps a copy of the pyramid.  Identical to
 * vv_octree_build_terrain.  VV_ERR_NODEV without that device. */
int vv_octree_build_terrain_gpu(const vv_terrain_desc* desc, int32_t device, vv_octree** out);
void vv_octree_destroy(vv_octree* tree);
int vv_octree_get_info(const vv_octree* tree, vv_octree_info* info);
/* Host mirror of the node pool in reference texture order, no brick resident
 * (2 * pool_dim product words). */
int vv_octree_node_words(const vv_octree* tree, uint32_t* words);
/* Node record for grid position (x,y,z): level (0 = root), mip-level voxel
 * origin of its brick region, constant flag, parent grid position. */
typedef struct vv_node_info {
    int32_t valid;
    int32_t level;
    int32_t origin[3];         /* brick origin in mip-level voxels (8*i)   */
    int32_t is_constant;
    int32_t has_children;
    int32_t parent[3];         /* -1 for the root */
} vv_node_info;
int vv_octree_node_info(const vv_octree* tree, uint32_t x, uint32_t y,
                        uint32_t z, vv_node_info* info);
/* Produce the stored 10^3 bricks of n nodes (given by grid position, 3
 * uint32 each) in `fmt` into `out` (n * 1000 texels).  This is
 * Node::copyMipMapToBrick (GigaVoxelsOctTree.cpp:1428-1488) over the mip
 * pyramid of GenerateMipMaps (:1030-1194). */
int vv_octree_produce_bricks(const vv_octree* tree, const uint32_t* xyz,
                             int32_t n, int32_t fmt, void* out);
/* The gradient bricks of the same nodes (the pGradientData half of
 * copyMipMapToBrick): leaf gradients are normalised central differences of
 * alpha with 0 outside the volume (VolumeDataSet::convert,
 * VolumeDataSet.cpp:144-209), coarser levels the box-filtered, renormalised
 * average of the level below (GenerateMipMap / GetBoxFilterAverage,
 * GigaVoxelsOctTree.cpp:809-960).  fmt VV_FMT_FP32 (float x, y, z, 0) or
 * VV_FMT_RGBA8 (round((g + 1) / 2 * 255) per component, for
 * gradients_unsigned).  Kept densely: trees of depth <= 6. */
int vv_octree_produce_gradients(const vv_octree* tree, const uint32_t* xyz,
                                int32_t n, int32_t fmt, void* out);
/* Dense mip level (RGBA8, x fastest) for checking on small volumes. */
int vv_octree_mip_level(const vv_octree* tree, int32_t level, uint32_t* out,
                        size_t out_words);
/* Column heights of the leaf level (dim*dim int32, x fastest).  This and
 * vv_octree_mip_level need a terrain tree (VV_ERR_ARG for a file tree). */
int vv_octree_heights(const vv_octree* tree, int32_t* out);

/* ---- GigaVoxels dataset files: .gvx / .gvb / .gvp ------------------------
 * A .gvx is the XML octree (a GigaVoxelsOctTree element with nested Node
 * elements, 8 children each, depth-first), voxels_<level>.gvb beside it the
 * level's bricks: int compressed, then per brick size_t dims[3], uint32
 * border[3], and colours and gradients as (int compressed, uint32 bytes,
 * payload).  A .gvp lists paged trees (OctTree elements with a TreeFile). */
enum {
    /* Store constant nodes' colours in their node words.  Without it a file
     * tree renders as the reference renders it: Node::setConstantValue
     * (GigaVoxelsOctTree.cpp:1611-1621) drops the colour, so constant nodes
     * are transparent black. */
    VV_GVX_CONSTANT_COLORS = 1,
    /* Skip the gradient payloads (GigaVoxelsReader::SetLoadNormals(false)). */
    VV_GVX_SKIP_GRADIENTS = 2
};
/* GigaVoxelsReader::LoadOctTreeFile (GigaVoxelsReader.cpp:373-514,541-563,
 * bricks :106-221).  The tree pages like a terrain tree through
 * vv_renderer_create; its bricks are kept on the host and, with
 * device_paging, in device memory, from where paging copies them into pool
 * slots.  A brick's node pointer is slot origin + the brick's border
 * (BrickPool::uploadBrick, GigaVoxelsBrickPool.cpp:800-808).  Supported:
 * brick size 8 (stored dims <= 10, border <= 2), uncompressed binary bricks,
 * MaxDepth <= 11.  Errors: VV_ERR_IO (missing or malformed file, or one the
 * reference rejects: depth or element mismatch, compression mismatch, empty
 * payload, data after the last brick), VV_ERR_ARG (unsupported content);
 * the message is in vv_last_error(NULL). */
int vv_octree_load_gvx(const char* path, int32_t flags, vv_octree** out);
/* Write tree.gvx and voxels_<level>.gvb into the existing directory `dir`,
 * in the voxelizer's layout (Voxelizer.cu:2840-3058,
 * VoxelBrickWriter.cu:509-818).  A terrain tree writes its 10^3 bricks with
 * a 1-voxel border and, for depth <= 6, its gradients (unsigned bytes); the
 * zero vector (128,128,128) otherwise or with VV_GVX_SKIP_GRADIENTS.  A file
 * tree writes back what it read. */
int vv_octree_save_gvx(const vv_octree* tree, const char* dir, int32_t flags);
typedef struct vv_gvx_info {
    int32_t file_backed;       /* 1 for a tree read from files */
    int32_t max_depth;         /* MaxDepth: levels */
    float origin[3];           /* X, Y, Z */
    float delta[3];            /* DeltaX.. */
    int32_t volume_size[3];    /* VolumeXSize.. */
    int32_t brick_size[3];     /* BrickXSize.. */
    int64_t bricks;            /* bricks held */
    int32_t has_gradients;     /* gradient payloads loaded (unsigned) */
    float ray_step_size;       /* getRayStepSize: one leaf voxel of the box */
} vv_gvx_info;
int vv_octree_gvx_info(const vv_octree* tree, vv_gvx_info* info);

/* One paged tree of a .gvp (PagedOctTreeNode, GigaVoxelsReader.cpp:59-96). */
typedef struct vv_gvp_tile {
    float center[3];
    float radius;
    float size_meters[3];
    char tree_file[1024];      /* read: the .gvp's directory joined; write: as given */
} vv_gvp_tile;
typedef struct vv_gvp_info {
    int32_t compressed;
    int32_t brick_size[3];
    int32_t tiles;             /* tiles in the file */
    float sphere_center[3];    /* BoundingSphere::expandBy over the tiles */
    double sphere_radius;      /* -1 with no tiles */
} vv_gvp_info;
/* LoadGVP (GigaVoxelsReader.cpp:35-101): the first min(cap, tiles) tiles. */
int vv_gvp_read(const char* path, vv_gvp_info* info, vv_gvp_tile* tiles, int32_t cap);
int vv_gvp_write(const char* path, const vv_gvp_info* info, const vv_gvp_tile* tiles, int32_t n);


/* ---- camera + uniform derivation ---------------------------------------- */

/* vox::Camera essentials (VoxVizCore/Camera.h). */
typedef struct vv_camera {
    float position[3];     /* normalized volume space */
    float look[3];         /* unit */
    float up[3];           /* unit, orthogonal to look */
    float fov_y_deg;       /* Camera default 45 (Camera.cpp:36) */
    float near_dist;
    int32_t width, height;
    int32_t frame;         /* Camera::getFrameCount */
} vv_camera;

/* Derive the draw uniforms exactly as GigaVoxelsRenderer::drawVolume
 * (GigaVoxelsRenderer.cpp:1630-1816) with the octree and the camera. */
int vv_compute_uniforms(const vv_octree_info* tree, const vv_camera* cam,
                        int32_t pool_slots_x, int32_t pool_slots_y,
                        int32_t pool_slots_z, float lod_scalar,
                        float alpha_stop, vv_uniforms* out);
/* Camera::getPixelSize (Camera.cpp:128-196). */
float vv_camera_pixel_size(const vv_camera* cam);
/* Seeded jitter texture values in [1,255] (size*size bytes). */
int vv_make_jitter(uint32_t seed, int32_t size, uint8_t* out);

/* ---- renderer: the plugin frame protocol -------------------------------- */

typedef struct vv_renderer vv_renderer;

typedef struct vv_renderer_desc {
    int32_t fmt;               /* brick pool format                        */
    int64_t pool_bytes;        /* brick pool budget (0 = all bricks fit)    */
    int32_t preload_all;       /* 1: make every brick resident at init      */
    int32_t request_cap;       /* compacted-list cap (0 = no cap)           */
    float lod_scalar;          /* 1.0 = one voxel per pixel                 */
    float alpha_stop;          /* 0.99 in the benchmark configs             */
    uint32_t jitter_seed;
    int32_t max_width, max_height;
    int32_t producer_threads;  /* host brick producers (0 = all cores)      */
    int32_t device_paging;     /* 1: de-duplicate requests and produce bricks
                                  on the GPU (same policy and results; the
                                  host keeps only the LRU list)             */
    int32_t color_rgba8;       /* 1: the frame's colour as RGBA8 unorm
                                  (VV_PASS_COLOR_RGBA8), 4 bytes per pixel;
                                  read_color then returns bytes             */
} vv_renderer_desc;

typedef struct vv_renderer_stats {
    int64_t frame;
    int64_t requests;          /* compacted entries this frame              */
    int64_t active_pixels;
    int64_t bricks_uploaded;   /* this frame                                */
    int64_t bricks_uploaded_total;
    int64_t resident_bricks;
    int64_t evictions_total;
    int32_t pool_slots;
    /* host wall time of the last update, milliseconds */
    float ms_readback;         /* request count + list read-back            */
    float ms_policy;           /* decode, dedupe, LRU                        */
    float ms_produce;          /* brick production on the host cores         */
    float ms_upload;           /* brick upload + node patches                */
    float ms_visit;            /* host pass over the distinct requested nodes
                                  (part of ms_readback with device paging)  */
    int32_t unique_nodes;      /* distinct requested nodes, last service     */
} vv_renderer_stats;

/* vox::Renderer lifecycle of the "gv" renderer (VoxVizCore/Renderer.h:20-110,
 * GigaVoxelsRenderer.cpp).  init: pools + initial bricks. */
int vv_renderer_create(vv_ctx* ctx, vv_octree* tree, const vv_renderer_desc* d,
                       vv_renderer** out);
void vv_renderer_destroy(vv_renderer* r);
/* draw(): ray cast + selection mask + histopyramid + compaction on device. */
int vv_renderer_draw(vv_renderer* r, const vv_camera* cam);
/* The frame protocol with postDraw kept apart, as GigaVoxelsRenderer splits
 * it: draw with `passes` VV_PASS_RAYCAST [| VV_PASS_COMPACT] (the selection
 * mask always runs: GigaVoxelsRenderer::draw, GigaVoxelsRenderer.cpp:
 * 1070-1088); vv_renderer_post_draw then runs the compaction of a frame
 * drawn without it (GigaVoxelsRenderer::postDraw -> compressNodeUsageList,
 * :1150-1186), and vv_renderer_update runs it itself if postDraw was not
 * called.  VV_ERR_ARG without VV_PASS_RAYCAST or with unknown bits. */
int vv_renderer_draw_passes(vv_renderer* r, const vv_camera* cam, int32_t passes);
int vv_renderer_post_draw(vv_renderer* r);
/* postDraw() + update(): read back the compacted page requests, run the
 * NodeUsageListProcessor / BrickPool::update policy (deterministic LRU),
 * produce and upload bricks and patch node words. */
int vv_renderer_update(vv_renderer* r);
/* The same page-request service for a compacted list drawn outside the
 * renderer (for example by vv_render_batch followed by vv_render with
 * VV_PASS_SELECT | VV_PASS_COMPACT): `requests` (device, 4 words per
 * entry), `count` (device, one word), at most `cap` entries read.  Needs
 * device_paging.  May be called for several views per frame. */
int vv_renderer_service(vv_renderer* r, const uint32_t* requests, const uint32_t* count, int32_t cap);
/* Deferred uploads (no counterpart in the reference, whose BrickPool::update
 * uploads at once): with `on`, update/service only choose bricks and node
 * words; vv_renderer_stage_uploads writes the frame's production jobs and
 * node patches to pinned mapped host memory and vv_renderer_enqueue_uploads
 * enqueues the device side on the context's stream.  The enqueued work reads
 * the staged counts on the device, so it can be captured once into a CUDA
 * graph and replayed every frame after staging.  The host must not stage
 * again until the previous enqueue (or replay) has completed. */
int vv_renderer_set_deferred(vv_renderer* r, int32_t on);
int vv_renderer_stage_uploads(vv_renderer* r);
int vv_renderer_enqueue_uploads(vv_renderer* r);
int vv_renderer_get_stats(const vv_renderer* r, vv_renderer_stats* out);
/* Device pointers of the last frame's buffers (valid until next draw). */
int vv_renderer_frame_buffers(vv_renderer* r, float** color, uint32_t** usage,
                              uint32_t** mask, uint32_t** requests,
                              uint32_t** request_count);
/* Copy the last frame's colour (H*W*4 floats) to host memory. */
int vv_renderer_read_color(vv_renderer* r, float* host_rgba);
/* The same copy on the renderer's copy stream, returning at once (no
 * counterpart in the reference, which blits on the GL thread).  The copy
 * starts when the page-request service (vv_renderer_update or _service)
 * has finished its read-outs, or at the next draw or wait, whichever comes
 * first, and overlaps the next draw (frames alternate between two colour
 * buffers; a draw waits only for the copy of the buffer it reuses).
 * `host_rgba` should be pinned and must stay valid until
 * vv_renderer_wait_readback returns. */
int vv_renderer_read_color_async(vv_renderer* r, float* host_rgba);
int vv_renderer_wait_readback(vv_renderer* r);
/* Copy the last frame's node-usage lists (H*W*12 words) and selection mask
 * (H*W words) to host memory; NULL skips a buffer.  This is the readback of
 * GigaVoxelsOctTree::updateNodeUsageListProcessor (GigaVoxelsOctTree.cpp:1852-1985)
 * for the raw lists, kept for checking. */
int vv_renderer_read_lists(vv_renderer* r, uint32_t* host_usage, uint32_t* host_mask);
/* Host copy of the compacted request list of the last update (n x 4 words). */
int vv_renderer_last_requests(const vv_renderer* r, uint32_t* out, int32_t cap,
                              int32_t* n);
/* Slot of every resident brick: out_xyz[i*3..] node grid position,
 * out_slot[i]; returns the count in *n. */
int vv_renderer_residency(const vv_renderer* r, uint32_t* out_xyz,
                          uint32_t* out_slot, int64_t cap, int64_t* n);
/* The brick pool's slots in LRU order, least recently used first: the order
 * of BrickPool::m_loadedBricks (GigaVoxelsBrickPool.h:66, moved by
 * notifyUsed GigaVoxelsBrickPool.cpp:406-424 and BrickPool::update :561-682),
 * which eviction takes from the front.  Writes min(cap, slots) entries and
 * the slot count to *n. */
int vv_renderer_lru_order(vv_renderer* r, uint32_t* out, int64_t cap, int64_t* n);
/* Uniforms of the last draw. */
int vv_renderer_last_uniforms(const vv_renderer* r, vv_uniforms* out);
vv_ctx* vv_renderer_ctx(vv_renderer* r);

/* ---- paged scenes: the tiles of a .gvp ------------------------------------
 * The reference's paged-scene path: each frame the cull visitor
 * (GigaVoxelsRenderer.cpp:667-798) tests every tile's bounding sphere
 * against the camera frustum (vox::Frustum, VoxVizCore/Frustum.cpp), stamps
 * visible tiles with the frame, requests loads of visible unloaded tiles
 * from the pager and lists the loaded ones farthest first (distance of the
 * centre to the near plane minus the radius); the list is drawn in order and
 * each tile blended over the colour with GL_SRC_ALPHA, GL_ONE_MINUS_SRC_ALPHA
 * (:997-1090).  The pager (GigaVoxelsDatabasePager.cpp) loads requests
 * sorted by last access (latest first) then distance (nearest first), merges
 * loaded trees at the next update and unloads tiles unseen for more than
 * stale_frames frames.  Each loaded tile is drawn by its own renderer (own
 * context, brick pool of pool_bytes_per_tile and LRU; the reference shares
 * one brick pool), with the camera mapped into the tile's box as drawVolume
 * maps it (the box must be a cube). */
typedef struct vv_scene vv_scene;
enum {
    VV_SCENE_HOST_ONLY = 1,    /* cull and page trees on the host; no drawing */
    VV_SCENE_SYNCHRONOUS = 2,  /* loads run inside vv_scene_update (no pager thread) */
    VV_SCENE_BATCHED = 4       /* the drawn tiles' ray casts as one batched launch
                                  (vv_render_batch); results are the same */
};
typedef struct vv_scene_desc {
    int32_t fmt;                  /* brick pool format of every tile */
    int64_t pool_bytes_per_tile;  /* 0: every brick of a tile fits */
    int32_t request_cap;          /* per tile (0: no cap) */
    float lod_scalar;             /* 0: 1.0 */
    float alpha_stop;             /* 0: 0.99 */
    uint32_t jitter_seed;
    int32_t device_paging;
    int32_t load_flags;           /* VV_GVX_* for every tile */
    int32_t stale_frames;         /* 0: 100, the reference's */
    float far_dist;               /* camera far plane; 0: 10000, vox::Camera's */
    int32_t flags;                /* VV_SCENE_* */
    int32_t reserved[4];
} vv_scene_desc;
typedef struct vv_scene_tile_state {
    int32_t loaded;               /* merged: drawn when visible */
    int32_t pending;              /* requested or loaded, not merged yet */
    int32_t visible;              /* inside the frustum at the last draw */
    int32_t drawn_order;          /* position in the last render list, -1 */
    int32_t failed;               /* its tree could not be loaded (not retried) */
    float dist_to_near_plane;     /* last draw; minus the radius when drawn */
    int64_t last_access;          /* frame of the last draw that saw it */
} vv_scene_tile_state;
typedef struct vv_scene_stats {
    int32_t tiles, loaded, pending, drawn;
    int64_t loads, unloads, load_failures;
    float load_ms_avg, load_ms_max;
} vv_scene_stats;
/* ctx: the context the scene's colour lives in (NULL with VV_SCENE_HOST_ONLY). */
int vv_scene_create(vv_ctx* ctx, const char* gvp_path, const vv_scene_desc* desc, vv_scene** out);
void vv_scene_destroy(vv_scene* scene);
/* Renderer::draw: cull, request loads, draw and blend.  The camera is in
 * world coordinates (the .gvp's and the trees' units). */
int vv_scene_draw(vv_scene* scene, const vv_camera* world_camera);
/* Renderer::update: merge loaded trees, unload stale tiles, then the
 * page-request service of every tile drawn by the last draw. */
int vv_scene_update(vv_scene* scene);
/* Block until the pager has no request left (loads still to be merged by
 * the next update). */
int vv_scene_wait_loads(vv_scene* scene);
int vv_scene_read_color(vv_scene* scene, float* host_rgba);
int vv_scene_tile_states(const vv_scene* scene, vv_scene_tile_state* out, int32_t cap);
int vv_scene_get_stats(const vv_scene* scene, vv_scene_stats* out);
/* The renderer of a loaded tile, owned by the scene (NULL otherwise); its
 * colour is the tile's FragColor before blending. */
vv_renderer* vv_scene_tile_renderer(vv_scene* scene, int32_t tile);

#ifdef __cplusplus
}
#endif

#endif /* VOXVIZ_B200_H */
