// Photon mapping with reference semantics (photon.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "refmode.hpp"

namespace rnb {

constexpr int kMaxPhotons = 1 << 22;

// Device scratch the photon mapper needs for n_photons photons.
cudaError_t photon_scratch_bytes(int n_photons, size_t &bytes);

// Both passes of renderPhotonMapped into argb (device, width*height 0xAARRGGBB).
// hp: host copy of the parameters (lights[0] emits); d_params: the same on the
// device. Synchronises st once (to size the deposit pass); deposits_out receives
// the number of stored photons.
cudaError_t launch_photon_mapped(const SceneView &sv, const float4 *ref_shade, const RefParams &hp,
                                 const RefParams *d_params, int n_photons, int gather_rays, void *scratch,
                                 size_t scratch_bytes, uint32_t *argb, int *status, cudaStream_t st,
                                 unsigned *deposits_out);

} // namespace rnb
