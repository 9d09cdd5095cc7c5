/* rednoise-b200: drop-in C ABI of the RedNoise renderer, served by CUDA kernels
 * for sm_100a (B200).
 *
 * Every declaration below keeps the symbol name, argument list, ownership and
 * return convention of the reference ABI it replaces, so a consumer built
 * against the reference header (C, ctypes, Rust FFI) links and behaves the same:
 *   reference header  include/rednoise/rednoise.h:1-54
 *   reference impl    src/capi.cpp:1-91
 * RN_PATHTRACED renders run on the GPU; there is no CPU fallback for them.
 */
#ifndef REDNOISE_H
#define REDNOISE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Reference version macros (include/rednoise/rednoise.h:16-18). */
#define RN_VERSION_MAJOR 0
#define RN_VERSION_MINOR 1
#define RN_VERSION_PATCH 2

/* Opaque scene: host triangles plus the lazily built device BVH and buffers. */
typedef struct rn_scene rn_scene;

/* Render modes, same values as the reference enum (rednoise.h:24).
 * Only RN_PATHTRACED is served by this library; the other modes return 0. */
typedef enum { RN_WIREFRAME = 0, RN_RASTERISED = 1, RN_RAYTRACED = 2, RN_PATHTRACED = 3 } rn_render_mode;

/* Load a Wavefront OBJ (+ its .mtl), scaling vertices by `scale`.
 * NULL on failure (missing file, malformed face, no faces).
 * Replaces rednoise.h:26-28 / capi.cpp:22-34. */
rn_scene *rn_scene_load_obj(const char *path, float scale);

/* Release a scene; NULL is ignored. Replaces rednoise.h:30-31 / capi.cpp:36-38. */
void rn_scene_free(rn_scene *scene);

/* Triangle count, 0 for NULL. Replaces rednoise.h:33-34 / capi.cpp:40-42. */
int rn_scene_triangle_count(const rn_scene *scene);

/* Render into the caller-owned RGBA8 buffer (width*height*4 bytes, row-major,
 * top row first) with the reference's fixed camera: position (0, 0, cam_z),
 * focal length 2.0 at scale 150, looking at the origin. For RN_PATHTRACED this
 * runs the reference path-tracer semantics (default disk light, depth 4,
 * per-pixel seeded sample stream, 8-bit clamp) on the GPU.
 * Returns 1 on success, 0 on invalid arguments, an unsupported mode or a
 * device failure (rn_pt_last_error() then holds the reason).
 * Replaces rednoise.h:36-41 / capi.cpp:44-79. */
int rn_render(const rn_scene *scene, rn_render_mode mode, int width, int height, float cam_z, int samples,
              unsigned char *rgba);

/* Write an RGBA8 buffer as a PNG. 1 on success, 0 on failure.
 * Replaces rednoise.h:43-45 / capi.cpp:81-85. */
int rn_save_png(const char *path, int width, int height, const unsigned char *rgba);

/* Library version string, "0.1.2" like the reference (capi.cpp:87-89). */
const char *rn_version(void);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* REDNOISE_H */
