// Bidirectional path tracing (renderBidirectional, src/BDPT.cpp) and primary-sample
// Metropolis light transport (renderMetropolis, src/Metropolis.cpp) on the GPU.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "traverse.cuh"

namespace rnb {

struct GiParams {
	int width, height;
	float position[3];
	float orient[9]; // camera axes right, up, backward (glm mat3 columns)
	float f;         // focalLength * scale, in pixels
	int samples;     // bidirectional: samples per pixel
	float exposure;
	unsigned long long seed;
	long long mutations; // Metropolis: total chain steps
	int chains;          // Metropolis: number of chains
	int bootstrap;       // Metropolis: bootstrap paths
};

constexpr int kBdptRecordSlots = 9;    // 4 camera vertices, the light point, 4 light vertices
constexpr int kBdptRecordBytes = 145;  // 9 x 16 B + the two subpath lengths
constexpr int kMltMaxBootstrap = 1 << 24;

// Bidirectional path tracing. reference_stream: the reference's std::mt19937 per image
// row (exact canvas; rows trace subpaths in stream order, pixels connect them in
// parallel, in column chunks of at most chunk_budget bytes of subpath records);
// otherwise Philox counter-based random numbers, subpaths one thread per sample.
size_t bdpt_scratch_bytes(const GiParams &p, bool reference_stream, size_t chunk_budget);
cudaError_t launch_bdpt(const SceneView &sv, const float4 *ref_shade, const GiParams &p, bool reference_stream,
                        size_t chunk_budget, void *scratch, uint32_t *argb, float *rgb, int *status, cudaStream_t st);

// Many-chain Metropolis sampler. rgb (may be null): the normalised radiance estimate
// (deposits x b x pixels / mutations) before exposure and tone mapping; b_out (may be
// null, device): the bootstrap mean luminance as a double.
size_t mlt_scratch_bytes(const GiParams &p);
cudaError_t launch_mlt(const SceneView &sv, const float4 *ref_shade, const GiParams &p, void *scratch, uint32_t *argb,
                       float *rgb, double *b_out, int *status, cudaStream_t st);

} // namespace rnb
