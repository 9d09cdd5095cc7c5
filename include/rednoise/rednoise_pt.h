/* rednoise-b200 additive path-tracing ABI (versioned, beside the drop-in
 * rednoise.h). These entry points have no counterpart in the reference's C ABI;
 * each one says which reference function's behaviour it exposes.
 *
 * Conventions
 *  - Every function returns rn_status; RN_OK is 0. On failure
 *    rn_pt_last_error() returns a message for the calling thread.
 *  - Array arguments are host pointers and calls are synchronous, unless
 *    `flags` contains RN_PT_DEVICE_POINTERS: then they are device pointers and
 *    the work is enqueued on `stream` (a cudaStream_t, NULL = the scene's own
 *    stream) without a host synchronisation.
 *  - Triangle indices are the caller's original indices.
 */
#ifndef REDNOISE_PT_H
#define REDNOISE_PT_H

#include <stdint.h>

#include "rednoise.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
	RN_OK = 0,
	RN_ERR_INVALID_ARGUMENT = 1,
	RN_ERR_CUDA = 2,
	RN_ERR_OUT_OF_MEMORY = 3,
	RN_ERR_UNSUPPORTED = 4,
	RN_ERR_DEVICE_TIMEOUT = 5,
	RN_ERR_CAPACITY = 6,
	RN_ERR_INTERNAL = 7
} rn_status;

/* flags */
#define RN_PT_DEVICE_POINTERS 1u /* arrays are device pointers; asynchronous on `stream` */
#define RN_PT_ORDER_NEAREST 2u   /* closest hit: nearest-child-first traversal (default: reference order) */
#define RN_PT_WIDTH2 4u          /* ray queries: traverse the 2-wide reference tree (default: its 4-wide collapse) */
#define RN_PT_WAVEFRONT_STATIC 8u /* wavefront: one ray per lane in the traversal stages (default: lanes refetch) */
#define RN_PT_RAY_SORT 16u        /* wavefront: bin each bounce's rays by origin cell and direction before tracing */
#define RN_PT_NO_RAY_SORT 32u     /* wavefront: never bin (default without either flag: the tuned choice) */
#define RN_PT_LBVH 64u            /* physical renders and ray queries: the GPU-built BVH (rn_pt_scene_build_lbvh),
                                     traversed nearest child first */

/* Physical-mode materials. */
#define RN_PT_LAMBERT 0
#define RN_PT_GGX 1
#define RN_PT_DIELECTRIC 2

/* A triangle scene given as arrays (all optional except vertices). The
 * reference fields feed the drop-in reference-mode renderer (ModelTriangle,
 * framework/ModelTriangle.h:26-39); the physical fields feed rn_pt_render. */
typedef struct {
	int num_triangles;
	const float *vertices;       /* 9 floats per triangle: v0, v1, v2 */
	const int *ref_rgb;          /* 3 ints per triangle, 0..255 (default 255) */
	const int *ref_material;     /* reference Material enum value (default Diffuse) */
	const float *ref_roughness;  /* reference Metal roughness (default 0.2) */
	const float *ref_normal;     /* 3 floats per triangle (default: cross(e0,e1)/|cross|) */
	const float *albedo;         /* 3 floats per triangle (default 0.8) */
	const float *emission;       /* 3 floats per triangle, radiance Le (default 0) */
	const int *material;         /* RN_PT_LAMBERT / RN_PT_GGX / RN_PT_DIELECTRIC (default Lambert) */
	const float *material_param; /* GGX alpha, or dielectric IOR (default 0.2 / 1.5) */
	const float *ref_vertex_normals; /* 9 floats per triangle, ModelTriangle::vertexNormals for the
	                                    ray-traced renderer's Phong/Gouraud shading (default: the face normal) */
} rn_pt_scene_desc;

/* Create a scene from arrays. The scene is freed with rn_scene_free. */
rn_status rn_pt_scene_create(const rn_pt_scene_desc *desc, rn_scene **out);

/* Build the reference BVH (src/BVH.cpp:6-63, identical tree and triangle
 * order) and upload the scene now instead of at the first query. */
rn_status rn_pt_scene_prepare(rn_scene *scene);

/* Build a second BVH on the GPU (a linear BVH: Morton codes, radix sort, Karras'
 * hierarchy, bottom-up boxes; one triangle per leaf) for callers that rebuild
 * often. Calls given RN_PT_LBVH use it with nearest-child-first traversal and ties
 * on the hit distance broken by leaf position: their closest hits agree with the
 * reference tree's except for exact ties and hits the reference's box test misses.
 * The reference tree stays the default. build_ms (may be NULL) receives the build
 * time including the upload of the vertices. Prepares the scene first. */
rn_status rn_pt_scene_build_lbvh(rn_scene *scene, void *stream, double *build_ms);

/* Facts about the prepared scene. */
typedef struct {
	int num_triangles;
	int internal_nodes;
	int depth;
	long long device_bytes;
	double build_ms;
} rn_pt_scene_info;
rn_status rn_pt_scene_get_info(rn_scene *scene, rn_pt_scene_info *out);

/* Dump the prepared BVH: order[n] (reference triangle order), and for each
 * reference node (count = internal + leaves) its box and links
 * (left, right, start, count) as BVH::Node holds them (src/BVH.h:22-26).
 * Query the node count with nodes == NULL. */
rn_status rn_pt_scene_dump_bvh(rn_scene *scene, int *order, int *node_count, float *bounds, int *links);

/* Copy the scene's triangles out (any pointer may be NULL): vertices (9 per
 * triangle), reference Colour (3 ints), reference Material and the face normal
 * as the loader computed it (src/ObjLoader.cpp:170-176). */
rn_status rn_pt_scene_get_triangles(const rn_scene *scene, float *vertices, int *ref_rgb, int *ref_material,
                                    float *ref_normal);

/* Closest hit for n rays (BVH::intersect, src/BVH.cpp:77-111): tri[i] is the
 * original index of the hit triangle or -1; t/u/v as the reference reports them
 * (t = +inf on a miss). ignore may be NULL (no triangle skipped). */
rn_status rn_pt_trace_closest(rn_scene *scene, int n, const float *origins, const float *directions, const int *ignore,
                              unsigned flags, void *stream, int *tri, float *t, float *u, float *v);

/* Any hit strictly before tmax[i] (BVH::occluded, src/BVH.cpp:113-139). */
rn_status rn_pt_trace_any(rn_scene *scene, int n, const float *origins, const float *directions, const float *tmax,
                          const int *ignore, unsigned flags, void *stream, int *occluded);

/* ---- reference-mode rendering (renderPathTraced, src/Renderer.cpp:1119-1170) ---- */

/* A light with the reference Light's fields and defaults (src/Light.h:13-29).
 * type: 0 point, 1 directional, 2 spot, 3 volume, 4 rectangle, 5 triangle. */
typedef struct {
	int type;
	float position[3];
	float direction[3];
	float colour[3];
	float intensity;
	float radius;
	float cone_cos;
	float atten_constant, atten_linear, atten_quadratic;
	float u_axis[3];
	float v_axis[3];
} rn_light;

/* Camera(width, height, focal_length, position) + lookAt(target) with the
 * reference's scale (src/Camera.h:13-25), plus renderPathTraced's arguments.
 * num_lights == 0 uses the reference's default light (a 0.15-radius disk at
 * (0, 0.95, 0), src/Renderer.cpp:1129-1134). max_depth is 4 in the reference. */
typedef struct {
	int width, height;
	float position[3];
	float target[3];
	float focal_length;
	float scale;
	int orthographic;
	float ortho_scale;
	int samples;
	int max_depth;
	int num_lights;
	const rn_light *lights;
	float aperture, focus_distance;
	float camera_motion[3];
	int aperture_blades;
} rn_pt_ref_params;

/* Defaults of rn_render: camera at (0, 0, cam_z) looking at the origin,
 * focal 2.0 x scale 150, depth 4, default light, no depth of field. */
void rn_pt_ref_params_init(rn_pt_ref_params *p, int width, int height, float cam_z, int samples);

/* Render with reference semantics. argb: width*height pixels in the reference
 * Canvas format 0xAARRGGBB (may be NULL); mean_rgb: optional width*height*3
 * floats of the per-pixel sample mean before the 8-bit clamp. */
rn_status rn_pt_render_reference(rn_scene *scene, const rn_pt_ref_params *params, unsigned flags, void *stream,
                                 uint32_t *argb, float *mean_rgb);

/* Shading models of the ray-traced renderer, in the reference's ShadingModel order. */
#define RN_PT_SHADING_FLAT 0
#define RN_PT_SHADING_GOURAUD 1
#define RN_PT_SHADING_PHONG 2

/* Whitted ray tracing with reference semantics (renderRaytraced,
 * src/Renderer.cpp:909-948, with traceRay / glassTrace / shadeDiffuse /
 * shadeSurface, src/Renderer.cpp:500-773): mirrors, glass (Fresnel-weighted
 * reflection and refraction), dispersive glass, tinted metal reflection, emissive
 * surfaces, and multi-light diffuse + specular shading with soft-shadow visibility
 * on an ambient floor. The camera, lights and max_depth (recursion levels, 0..8;
 * the reference uses 4) come from params; samples and the depth-of-field fields
 * are not used. fog_density > 0 blends towards fog_colour (NULL: the reference's
 * default (200, 210, 230)) by 1 - exp(-density * distance). argb: width*height
 * pixels 0xAARRGGBB. rn_render(RN_RAYTRACED) is this call with Phong shading. */
rn_status rn_pt_render_raytraced(rn_scene *scene, const rn_pt_ref_params *params, int shading, float fog_density,
                                 const float *fog_colour, unsigned flags, void *stream, uint32_t *argb);

/* Photon mapping with reference semantics (renderPhotonMapped,
 * src/Renderer.cpp:1177-1349, PhotonMap, src/Photon.cpp): num_photons photons
 * (the reference's default is 200000) from the first light, traced through
 * mirrors, metal and glass and stored at diffuse hits with Russian roulette, all
 * drawn from one std::mt19937(777) stream in the reference's order; then per pixel
 * direct light plus the irradiance gathered within 0.25 units (gather_rays > 0: a
 * final gather of that many cosine rays, each image row drawing from
 * std::mt19937(1000 + y)). The camera and lights come from params (samples,
 * max_depth and depth-of-field fields are not used). argb: width*height pixels
 * 0xAARRGGBB; num_stored (may be NULL) receives the number of stored photons. */
rn_status rn_pt_render_photon_mapped(rn_scene *scene, const rn_pt_ref_params *params, int num_photons, int gather_rays,
                                     unsigned flags, void *stream, uint32_t *argb, unsigned *num_stored);

/* Testing hook, no reference counterpart: after `after` more successful device
 * allocations the next one fails as if the device were out of memory (the call
 * that made it returns RN_ERR_OUT_OF_MEMORY), once; after < 0 turns it off. For
 * checking that every call fails cleanly and the library stays usable after a
 * failed allocation. Process-wide; not for use while other threads render. */
rn_status rn_pt_inject_allocation_failure(long long after);

/* Random-number streams of rn_pt_render_bidirectional. */
#define RN_PT_RNG_REFERENCE 0 /* the reference's std::mt19937(9871 + y) per image row: the reference's canvas */
#define RN_PT_RNG_COUNTER 1   /* Philox-4x32-10 per (pixel, sample) under `seed`: same estimator, fully parallel */

/* Bidirectional path tracing with reference semantics (renderBidirectional,
 * src/BDPT.cpp:65-144): per sample a camera subpath and a subpath from the fixed
 * 0.36 x 0.36 ceiling emitter at (0, 0.33, 0) (Le = 30), both diffuse with up to four
 * bounces, every camera vertex connected to every light vertex with a shadow ray and
 * the uniform MIS weight 1 / (i + j + 2); then exposure, Reinhard and the 8-bit
 * canvas. The reference's defaults are samples = 64, exposure = 40. Only the camera
 * fields of params are used (width, height, position, target, focal_length, scale).
 * argb: width*height pixels 0xAARRGGBB; rgb (may be NULL): width*height*3 floats,
 * accum * exposure / samples before tone mapping. seed is used by RN_PT_RNG_COUNTER. */
rn_status rn_pt_render_bidirectional(rn_scene *scene, const rn_pt_ref_params *params, int samples, float exposure,
                                     int rng, unsigned long long seed, unsigned flags, void *stream, uint32_t *argb,
                                     float *rgb);

/* Primary-sample-space Metropolis light transport with reference semantics
 * (renderMetropolis, src/Metropolis.cpp:85-192): the reference's diffuse path
 * tracer with next-event estimation to the same emitter as a function of its random
 * numbers, a bootstrap of `bootstrap` paths for the normalisation (the reference uses
 * 100000), and `mutations` Markov-chain steps in total (reference default 4000000)
 * with the reference's large-step (p = 0.3) and Gaussian small-step (sigma = 0.02)
 * mutations, acceptance and expected-value deposits; exposure (reference default 16)
 * and Reinhard onto the canvas. The steps are split over `chains` chains run in
 * parallel (0: mutations / 16, at most 2097152), each started from a bootstrap path
 * drawn in proportion to its luminance; random numbers are Philox streams under
 * `seed`. argb: width*height pixels; rgb (may be NULL): width*height*3 floats of
 * the normalised radiance estimate before exposure; mean_luminance (may be NULL): the
 * bootstrap's mean luminance b. Only the camera fields of params are used. */
rn_status rn_pt_render_metropolis(rn_scene *scene, const rn_pt_ref_params *params, long long mutations, float exposure,
                                  int chains, int bootstrap, unsigned long long seed, unsigned flags, void *stream,
                                  uint32_t *argb, float *rgb, double *mean_luminance);

/* ---- canvas post-processing (src/Renderer.cpp:1353-1470), reference semantics ----
 * Canvases are width*height pixels 0xAARRGGBB, processed in place; host arrays
 * unless flags has RN_PT_DEVICE_POINTERS. */

/* toneMap: Reinhard on exposure-scaled colour, then gamma. */
rn_status rn_pt_tonemap(uint32_t *argb, int width, int height, float exposure, float gamma, unsigned flags,
                        void *stream);
/* applyBloom: pixels brighter than threshold (luma in 0..1), blurred by three
 * separable 13-tap box passes, added back times intensity. */
rn_status rn_pt_bloom(uint32_t *argb, int width, int height, float threshold, float intensity, unsigned flags,
                      void *stream);
/* applyFXAA: interior pixels on luma edges (contrast >= 0.12) blended towards
 * their 4-neighbour average. */
rn_status rn_pt_fxaa(uint32_t *argb, int width, int height, unsigned flags, void *stream);
/* AccumBuffer::add / resolve: sum (3 floats per pixel, read and written) += the
 * canvas colour; resolve writes sum / count as a canvas. */
rn_status rn_pt_accum_add(float *sum, const uint32_t *argb, int width, int height, unsigned flags, void *stream);
rn_status rn_pt_accum_resolve(const float *sum, int count, uint32_t *argb, int width, int height, unsigned flags,
                              void *stream);

/* Copy the scene's per-corner vertex normals out (9 floats per triangle), as the
 * reference OBJ loader smooths them (src/ObjLoader.cpp:178-204). */
rn_status rn_pt_scene_get_vertex_normals(const rn_scene *scene, float *vertex_normals);

/* ---- physical-mode rendering (the additive path-tracing estimator) ---- */

/* Pinhole camera looking from `position` at `target`, vertical field of view. */
typedef struct {
	float position[3];
	float target[3];
	float up[3];
	float vfov_deg;
	int width, height;
} rn_pt_camera;

#define RN_PT_AUTO 0
#define RN_PT_MEGAKERNEL 1
#define RN_PT_WAVEFRONT 2

/* spp samples per pixel, indices [sample_offset, sample_offset + spp); paths
 * have at most max_depth scattering vertices; Russian roulette from vertex
 * rr_depth (>= max_depth disables it); env is the radiance of escaping rays. */
typedef struct {
	int spp;
	int max_depth;
	int rr_depth;
	int integrator; /* RN_PT_AUTO / RN_PT_MEGAKERNEL / RN_PT_WAVEFRONT */
	unsigned long long seed;
	unsigned sample_offset;
	float env[3];
} rn_pt_settings;

/* Render and write the per-pixel mean radiance (width*height*3 floats, RGB,
 * row-major, top row first) to rgb. Next-event estimation to emissive triangles,
 * Lambert / GGX / dielectric sampling and Russian roulette (rednoise_b200's
 * physical estimator; the reference's renderPathTraced loop structure,
 * src/Renderer.cpp:1119-1170, with float accumulation instead of 8 bits). */
rn_status rn_pt_render(rn_scene *scene, const rn_pt_camera *camera, const rn_pt_settings *settings, unsigned flags,
                       void *stream, float *rgb);

/* Add the per-pixel SUM of samples [sample_offset, sample_offset + spp) to
 * accum (width*height*3 floats, read and written). Samples are added in index
 * order, so splitting a render over calls reproduces one call bit for bit (a
 * resumable progressive render). */
rn_status rn_pt_render_accumulate(rn_scene *scene, const rn_pt_camera *camera, const rn_pt_settings *settings,
                                  unsigned flags, void *stream, float *accum);

/* Maximum image size of rn_pt_render_static, in pixels (512 x 512). */
#define RN_PT_STATIC_MAX_PIXELS 262144

/* rn_pt_render without memory allocation, for callers that may not allocate
 * while they render (a host that owns a fixed memory budget, a framework whose
 * allocator must not be bypassed, a real-time loop). No counterpart in the
 * reference, which renders on the CPU into its own buffers. Runs the megakernel
 * (settings->integrator is ignored) with its per-pixel sums and work counter in
 * a fixed array inside the library (RN_PT_STATIC_MAX_PIXELS * 12 + 256 bytes on
 * each GPU) and writes the mean radiance to rgb, a DEVICE pointer of
 * width*height*3 floats, asynchronously on stream (NULL: the scene's stream).
 * The scene must be prepared (rn_pt_scene_prepare) and its device current.
 * Larger images return RN_ERR_CAPACITY; an rgb that is not device or managed
 * memory of the scene's GPU returns RN_ERR_INVALID_ARGUMENT, both before any GPU
 * work. The first call on a device looks up the array's address and keeps it;
 * make it before any stream capture, and do not call this after cudaDeviceReset
 * of that device. All calls share the array: calls whose GPU work overlaps race
 * and must be serialised by the caller. A traversal error is reported by the
 * scene's next synchronising call. */
rn_status rn_pt_render_static(rn_scene *scene, const rn_pt_camera *camera, const rn_pt_settings *settings,
                              unsigned flags, void *stream, float *rgb);

/* ---- autotuning ---- */

/* Result of rn_pt_autotune: the chosen integrator and samples per wave (the
 * wavefront's path-queue capacity in samples of every pixel), with the measured
 * throughput of each candidate. */
typedef struct {
	int integrator;        /* RN_PT_MEGAKERNEL or RN_PT_WAVEFRONT */
	int samples_per_wave;  /* wavefront queue capacity = width*height*samples_per_wave paths */
	double megakernel_sps; /* samples per second of the megakernel */
	double wavefront_sps;  /* samples per second of the best wavefront configuration */
	int dynamic_fetch;     /* wavefront traversal stages hand new rays to lanes whose ray finished */
	int ray_sort;          /* wavefront bins each bounce's rays by origin cell and direction */
} rn_pt_tuning;

/* Time short renders of this scene/camera/settings (a few samples per pixel)
 * with the megakernel and with the wavefront at several queue capacities, keep
 * the fastest, and remember it for RN_PT_AUTO renders of the same scene and
 * image size. `out` may be NULL. */
rn_status rn_pt_autotune(rn_scene *scene, const rn_pt_camera *camera, const rn_pt_settings *settings, unsigned flags,
                         rn_pt_tuning *out);

/* ---- profiling ---- */

/* Device time of each stage kind of one wavefront frame, summed over the frame's
 * bounces and waves (milliseconds), from CUDA events recorded between the stages. */
typedef struct {
	double camera_ms;      /* camera rays */
	double ray_sort_ms;    /* counting sorts of the closest-hit queues */
	double extend_ms;      /* closest hits */
	double shade_ms;       /* shading, next-event records, continuations */
	double shadow_sort_ms; /* counting sorts of the shadow records */
	double shadow_ms;      /* any hits of the shadow records */
	double accumulate_ms;  /* per-pixel sums and the resolve to the mean image */
	double total_ms;       /* the whole frame */
	int launches;          /* kernels launched */
	int waves;             /* waves of the frame */
	int samples_per_wave;  /* the wavefront configuration that ran */
	int dynamic_fetch;
	int ray_sort;
} rn_pt_stage_times;

/* One frame of rn_pt_render through the wavefront integrator, with the
 * configuration an RN_PT_AUTO render of these settings would use when its tuned
 * choice is the wavefront (else the wavefront's defaults; RN_PT_RAY_SORT /
 * RN_PT_NO_RAY_SORT / RN_PT_WAVEFRONT_STATIC in flags apply as for rn_pt_render),
 * launched kernel by kernel instead of from the captured frame graph with an
 * event after every stage, so each stage's device time can be measured. rgb
 * receives the mean image (a device pointer when flags has RN_PT_DEVICE_POINTERS,
 * else host memory); it equals rn_pt_render's. Synchronises the stream. A
 * profiling aid with no counterpart in the reference. */
rn_status rn_pt_profile_wavefront(rn_scene *scene, const rn_pt_camera *camera, const rn_pt_settings *settings,
                                  unsigned flags, void *stream, float *rgb, rn_pt_stage_times *out);

/* Read the device buffer buf (bytes, 16-byte aligned) `passes` times per launch,
 * `launches` times, with 16-byte loads from a persistent grid, after one untimed
 * launch, and write the device time of the timed launches to *ms (bandwidth =
 * bytes * passes * launches / ms). l2_only: the loads bypass L1, so a buffer well
 * under the L2's size gives the L2 read bandwidth and one far above it the HBM
 * read bandwidth. Synchronises the stream. A roofline probe with no counterpart in
 * the reference. */
rn_status rn_pt_probe_read(const void *buf, size_t bytes, int passes, int launches, int l2_only, void *stream,
                           float *ms);

/* ---- differentiable rendering ---- */

/* Overwrite per-triangle albedo (3 floats per triangle) and / or emitted
 * radiance (3 floats per triangle; only triangles that were emitters when the
 * scene was prepared keep emitting). Either pointer may be NULL. */
rn_status rn_pt_scene_set_materials(rn_scene *scene, const float *albedo, const float *emission, unsigned flags,
                                    void *stream);

/* Path-replay adjoint of rn_pt_render over n_views camera views of one scene:
 * given d_images[v] = dL/d(mean image of view v) (width*height*3 floats), write
 * d_albedo = dL/d(albedo) and d_emission = dL/d(emitted radiance), 3 floats per
 * triangle each (overwritten; either may be NULL). Each view's settings give its
 * adjoint samples (spp, seed, sample_offset, depth, roulette). Every path is
 * regenerated from its RNG key and traced again. settings->integrator picks the
 * schedule: RN_PT_MEGAKERNEL (one thread per path, memory O(pixels)),
 * RN_PT_WAVEFRONT (waves of paths binned like rn_pt_render's wavefront; each path
 * in flight keeps its continuation vertices, 32 bytes per vertex), RN_PT_AUTO
 * (waves for scenes above 4096 triangles). Roulette probabilities are treated as
 * constants. */
rn_status rn_pt_backward(rn_scene *scene, int n_views, const rn_pt_camera *cameras, const rn_pt_settings *settings,
                         const float *const *d_images, unsigned flags, void *stream, float *d_albedo,
                         float *d_emission);

/* ---- batched rendering: many scenes / cameras / resolutions in one launch ---- */

typedef struct rn_pt_batch rn_pt_batch;

/* One job: a scene seen through a camera with its own settings (spp, depth,
 * seed, sample_offset; the integrator field is ignored, the batch's applies). */
typedef struct {
	rn_scene *scene;
	rn_pt_camera camera;
	rn_pt_settings settings;
} rn_pt_job;

/* Build a batch. RN_PT_WAVEFRONT packs every job's paths into one wave
 * schedule whose whole frame is captured once as a CUDA graph and replayed;
 * RN_PT_MEGAKERNEL renders the jobs one megakernel launch after another;
 * RN_PT_AUTO lets the autotuner choose. flags: RN_PT_ORDER_NEAREST. The batch
 * keeps pointers to the scenes, which must outlive it. */
rn_status rn_pt_batch_create(const rn_pt_job *jobs, int n, int integrator, unsigned flags, rn_pt_batch **out);

/* Render every job once. sample_offset is added to each job's own offset
 * (progressive frames). out[j] receives job j's mean radiance, width*height*3
 * floats; with RN_PT_DEVICE_POINTERS the out[j] are device pointers and the
 * work is enqueued on `stream` without a host synchronisation. */
rn_status rn_pt_batch_render(rn_pt_batch *batch, unsigned sample_offset, unsigned flags, void *stream,
                             float *const *out);

/* The integrator the batch runs (after RN_PT_AUTO was resolved). */
int rn_pt_batch_integrator(const rn_pt_batch *batch);

void rn_pt_batch_free(rn_pt_batch *batch);

/* Profiling counters of the reference traversal algorithm (src/BVH.cpp:77-139,
 * box tests counted when a node is popped) over the rays of one render with
 * these settings: counters[7] = samples, closest queries, any-hit queries,
 * closest box tests, closest triangle tests, any-hit box tests, any-hit
 * triangle tests. 24 B per box test and 36 B per triangle test are the
 * algorithmic bytes of a query. */
rn_status rn_pt_count_traversal(rn_scene *scene, const rn_pt_camera *camera, const rn_pt_settings *settings,
                                long long *counters);

/* Message for the last failure on this thread ("" if none). */
const char *rn_pt_last_error(void);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* REDNOISE_PT_H */
