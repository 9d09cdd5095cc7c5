// Path-replay adjoint kernels (adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include "physical.cuh"

namespace rnb {

// One camera view of the adjoint: its settings and the gradient of the loss
// with respect to its mean image (3 floats per pixel, device memory).
struct AdjView {
	PhysCamera cam;
	PhysSettings st;
	const float *dimg;
	int n_pix;
	unsigned item_base; // first (pixel, sample) work item of the view: sum of n_pix * spp before it
};

// Scenes up to this many triangles accumulate their gradients in shared memory.
constexpr int kAdjointSharedTris = 4096;

// counter: one device word, the work counter (zeroed on the stream here).
cudaError_t launch_adjoint(const PhysScene &sc, const AdjView *d_views, int n_views, unsigned total_items,
                           float *d_alb, float *d_em, int n_tris, unsigned *counter, int *status, cudaStream_t st);

// Overwrite per-triangle albedo and / or emitted radiance of the shading records.
cudaError_t launch_set_materials(float4 *shade, int n, const float *albedo, const float *emission, cudaStream_t st);

} // namespace rnb
