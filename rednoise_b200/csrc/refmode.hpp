// Parameters of the reference-mode renderer (renderPathTraced semantics).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "traverse.cuh"

namespace rnb {

// Light types, same order as the reference's LightType (src/Light.h:8).
enum RefLightType : int {
	kLightPoint = 0,
	kLightDirectional = 1,
	kLightSpot = 2,
	kLightVolume = 3,
	kLightRectangle = 4,
	kLightTriangle = 5,
};

// Mirrors the fields of the reference Light (src/Light.h:13-29).
struct RefLight {
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
};

constexpr int kMaxRefLights = 16;
constexpr int kMaxRefDepth = 15;

struct RefParams {
	int width, height;
	float position[3];
	float orient[9]; // camera axes right, up, backward (glm mat3 columns)
	float f;         // focalLength * scale, in pixels
	int orthographic;
	float ortho_scale;
	int samples;
	int max_depth;
	int num_lights;
	RefLight lights[kMaxRefLights];
	float aperture, focus_distance;
	float camera_motion[3];
	int aperture_blades;
	int aperture_args_right_to_left;
	// ray-traced renderer only
	int shading; // 0 flat, 1 Gouraud, 2 Phong
	float fog_density;
	float fog_colour[3];
};

constexpr int kMaxWhittedDepth = 8;

// Whitted ray tracing (renderRaytraced). ref_geom: 6 float4 per triangle in the
// caller's triangle order: v0, v1, v2, then the three vertex normals.
cudaError_t launch_render_raytraced(const SceneView &sv, const float4 *ref_shade, const float4 *ref_geom,
                                    const RefParams *d_params, int width, int height, uint32_t *argb, int *status,
                                    cudaStream_t st);

// Shadow rays a light's visibility pattern casts (src/Renderer.cpp:390-498).
__host__ __device__ inline int ref_tap_count(const RefLight &L) {
	if (L.type == kLightDirectional)
		return 1;
	if (L.type == kLightRectangle || L.type == kLightTriangle)
		return 9;
	if (L.radius <= 0.0f)
		return 1;
	return L.type == kLightVolume ? 12 : 9;
}

// The drop-in path tracer (renderPathTraced semantics) in three passes: paths,
// shadow rays, fold. Scratch: at least ref_defer_bytes_per_pixel(p) +
// kRefDeferFixedBytes; larger images run in pixel chunks that fit.
constexpr size_t kRefDeferFixedBytes = 256 + (size_t(4) << 15) + 2048;
size_t ref_defer_bytes_per_pixel(const RefParams &p);
cudaError_t launch_render_reference(const SceneView &sv, const float4 *ref_shade, const RefParams &p,
                                    const RefParams *d_params, uint32_t *argb, float *mean_rgb, int *status,
                                    void *scratch, size_t scratch_bytes, cudaStream_t st);

} // namespace rnb
