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
	int pix_base; // first global pixel index of the view
};

// Scenes up to this many triangles accumulate their gradients in shared memory.
constexpr int kAdjointSharedTris = 4096;

cudaError_t launch_adjoint(const PhysScene &sc, const AdjView *d_views, int n_views, int total_pix, float *d_alb,
                           float *d_em, int n_tris, int *status, cudaStream_t st);

// Overwrite per-triangle albedo and / or emitted radiance of the shading records.
cudaError_t launch_set_materials(float4 *shade, int n, const float *albedo, const float *emission, cudaStream_t st);

} // namespace rnb
