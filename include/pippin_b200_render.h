/* pippin_b200: batched rasteriser of environment poses into RGBA8, linear
 * depth and geom-id segmentation, one image per (environment, view).
 *
 * Replaces the reference's Metal renderer behind the `Renderer` trait
 * (crates/pippin-env/src/lib.rs:220-238): `MetalRenderer::new(scene, config)`
 * (crates/pippin-render/src/lib.rs:95-170) becomes pg_render_create with the
 * scene already triangulated (the triangle meshes of
 * crates/pippin-render/src/mesh.rs, built by the host mirror), and
 * `MetalRenderer::render(slot, nenv, geoms, cams, appearance)`
 * (crates/pippin-render/src/lib.rs:234-355) becomes pg_render_frames (host
 * buffers) or pg_render_frames_device (device buffers, asynchronous on the
 * renderer's stream). The shading is that of
 * crates/pippin-render/src/render.metal:67-145.
 *
 * Layouts (all little-endian, row-major):
 *   vertex   8 words: pos f32[3], geom u32, normal f32[3], flags u32 (bit 0:
 *            checker pattern); the two u32 are stored in f32 slots by bits.
 *   triangle 3 u32 vertex indices, drawn in array order.
 *   view     16 f32: scene camera index (as f32; -1 = fixed pose), fx =
 *            f / aspect, fy = f, pad, then the fixed pose (pos[3], mat[9]);
 *            f = 1 / tan(fovy / 2).
 *   pose     12 f32: pos[3], row-major mat[9] (lib.rs:102-107).
 *   appearance 8 f32: rgba[4], scale[3], pad (lib.rs:160-166); alpha <= 0
 *            hides the geom in that environment.
 *   uniforms 8 f32: near, far, A = far / (near - far), A * near, the key
 *            light direction (unit, camera space) [3], pad.
 *   outputs  (env, view, y, x): rgba u8[4], depth f32 (linear, `far` on the
 *            background), segmentation i32 (geom id, -1 on the background).
 *
 * Every function returns 0 on success or a PG_ERR_* code (pippin_b200.h),
 * with the message in pg_last_error(). */
#ifndef PIPPIN_B200_RENDER_H
#define PIPPIN_B200_RENDER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pg_renderer pg_renderer;

#define PG_RENDER_VERTEX_WORDS 8
#define PG_RENDER_VIEW_WORDS 16
#define PG_RENDER_POSE_WORDS 12
#define PG_RENDER_APPEARANCE_WORDS 8

/* Uploads the triangulated scene and the view table to `device`.
 * base_appearance (ngeom x 8) is used when a frame supplies none. At most
 * 4096 views; a frame renders fewer than 2^31 images (nenv x nview), else
 * PG_ERR_UNSUPPORTED here or PG_ERR_INVALID from the frame calls. */
int pg_render_create(const float* vertices, int64_t nvert, const uint32_t* triangles, int64_t ntri, int64_t ngeom,
                     int64_t ncam, const float* views, int64_t nview, const float* base_appearance, int64_t width,
                     int64_t height, const float* uniforms, int device, pg_renderer** out);

int pg_render_destroy(pg_renderer* r);

/* Renders nenv environments from host buffers: geoms (nenv x ngeom poses),
 * cams (nenv x ncam poses; may be NULL when ncam is 0), appearance (nenv x
 * ngeom, or NULL for the scene's colours at unit scale). Writes host outputs
 * of nenv x nview x height x width pixels and returns when they are written.
 * The *_len arguments are element counts, checked against nenv. */
int pg_render_frames(pg_renderer* r, int64_t nenv, const float* geoms, size_t geoms_len, const float* cams,
                     size_t cams_len, const float* appearance, size_t appearance_len, uint8_t* rgba, float* depth,
                     int32_t* seg);

/* The same from device buffers into device outputs, enqueued on the
 * renderer's stream without waiting. */
int pg_render_frames_device(pg_renderer* r, int64_t nenv, const float* geoms, const float* cams,
                            const float* appearance, uint8_t* rgba, float* depth, int32_t* seg);

/* The renderer's CUDA stream (a cudaStream_t). */
void* pg_render_stream(const pg_renderer* r);

int pg_render_synchronize(pg_renderer* r);

#ifdef __cplusplus
}
#endif

#endif
