// Launchers of the physical-mode kernels.
#pragma once

#include <cuda_runtime.h>

#include "physical.cuh"

namespace rnb {

// Megakernel: accum (3 floats per pixel) += sum of samples [offset, offset + spp).
cudaError_t launch_megakernel(const PhysScene &sc, const PhysCamera &cam, const PhysSettings &st, float *accum,
                              unsigned *counter, int *status, cudaStream_t stream);

// Reference-order traversal counters over a frame (7 counters, see megakernel.cu).
cudaError_t launch_count(const PhysScene &sc, const PhysCamera &cam, const PhysSettings &st, unsigned long long *out,
                         int *status, cudaStream_t stream);

// mean = accum / total_spp (3 floats per pixel).
cudaError_t launch_resolve(const float *accum, float *mean, long n_floats, float inv_spp, cudaStream_t stream);

} // namespace rnb
