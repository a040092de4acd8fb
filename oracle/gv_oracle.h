/* gv_oracle.h - C interface of the CPU oracle (test infrastructure only).
 * Loaded by tests/, the smoke check and the cpu_baseline leg of bench.py. */
#ifndef GV_ORACLE_H
#define GV_ORACLE_H
#include <stdint.h>
#include "../include/voxviz_b200.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_scene {
    const uint32_t* nodes;  /* node pool, reference texture order, 2 words/texel */
    int32_t node_dim[3];
    const void* bricks;     /* brick pool, slot-major brick-linear texels */
    int32_t fmt;            /* vv_fmt */
    int32_t slots[3];
    const uint8_t* jitter;  /* jitter_tex_size^2 values */
    const void* grads;      /* gradient pool, same slots (lighting), or NULL */
    int32_t grad_fmt;       /* VV_FMT_FP32 or VV_FMT_RGBA8 */
} oracle_scene;

/* Rows [row0,row1) of the ray cast.  precision 32: float colour (4 floats per
 * pixel), 64: double colour.  usage: 12 words per pixel (may be NULL). */
int oracle_raycast(const vv_uniforms* u, const oracle_scene* s, int precision, int row0, int row1,
                   void* color, uint32_t* usage, int threads, int32_t* status);
int oracle_max_iterations(const vv_uniforms* u);
/* The RGBA8 texels (1000 per brick) of `bricks` DXT5 or DXT1 pool slots
 * (90 blocks each), decoded as the oracle's texture fetch decodes them. */
int oracle_dxt_decode(const void* blocks, int fmt, long long bricks, uint32_t* rgba8);
/* oracle_raycast plus `trace` (one uint64 per pixel of the full image, may
 * be NULL): a hash of each pixel's control flow (fragment, inside test, per
 * leaf segment the node, depth, flags, step count and samples composited,
 * then the iteration count).  Equal traces in the binary32 and binary64 runs
 * mean the same decisions were taken. */
int oracle_raycast_trace(const vv_uniforms* u, const oracle_scene* s, int precision, int row0, int row1,
                         void* color, uint32_t* usage, uint64_t* trace, int threads, int32_t* status);
/* The binary32 ray cast's sample sequence from `traj` re-evaluated in
 * binary64 with texel values from `vals` (same layout): 4 doubles per pixel
 * for rows [row0,row1) of a full-image buffer. */
int oracle_fixed_path(const vv_uniforms* u, const oracle_scene* traj, const oracle_scene* vals, int row0,
                      int row1, double* color, int threads);
/* Adjoint of the binary32 ray cast with binary64 accumulation: ADDS
 * dL/d(texel) (4 doubles per pool texel, slot-major) for rows [row0,row1)
 * given dL/d(colour) (4 floats per pixel).  Single-threaded. */
int oracle_backward(const vv_uniforms* u, const oracle_scene* s, const float* dl_dcolor, double* grad,
                    int row0, int row1);
/* oracle_backward, and when grad_abs is not NULL also ADDS to it the same
 * sums over absolute values (|w| * |T| * |g| with g's alpha recurrence run
 * on absolute values): per texel the magnitude of the terms whose sum is the
 * gradient.  A lower-precision implementation's rounding error is bounded
 * by a small multiple of its unit roundoff times this magnitude. */
int oracle_backward_bound(const vv_uniforms* u, const oracle_scene* s, const float* dl_dcolor, double* grad,
                          double* grad_abs, int row0, int row1);
int oracle_select(const uint32_t* usage, int w, int h, uint32_t* mask);
int oracle_compress(const uint32_t* usage, const uint32_t* mask, int w, int h, int max_push, int cap,
                    uint32_t* out, uint32_t* total);

#ifdef __cplusplus
}
#endif
#endif
