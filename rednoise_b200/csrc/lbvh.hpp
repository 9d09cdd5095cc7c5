// The GPU-built linear BVH (lbvh.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace rnb {

struct LbvhResult {
	float root_lo[3], root_hi[3];
	int root_ref;
	int internal_nodes;
	int depth; // leaf depth, root = 1
};

// Device scratch for n triangles.
size_t lbvh_scratch_bytes(int n);

// Build from d_v9 (9 floats per triangle, device). d_nodes: 4 float4 per internal
// node (n - 1); d_tris: 3 float4 per triangle, in leaf order (2-wide device layout).
// Synchronises st once at the end (root box and depth).
cudaError_t lbvh_build(const float *d_v9, int n, void *scratch, size_t scratch_bytes, float4 *d_nodes,
                       float4 *d_tris, LbvhResult &res, cudaStream_t st);

} // namespace rnb
