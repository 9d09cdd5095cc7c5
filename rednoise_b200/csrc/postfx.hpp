// Canvas post-processing kernels with reference semantics (postfx.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rnb {

constexpr int kPostBlurRadius = 6; // applyBloom's box radius (src/Renderer.cpp:1404)

// All canvases are device arrays of 0xAARRGGBB pixels.
cudaError_t postfx_tonemap(uint32_t *px, long n, float exposure, float gamma, cudaStream_t st);
// bright / tmp: n float3 of scratch each.
cudaError_t postfx_bloom(uint32_t *px, int W, int H, float threshold, float intensity, float3 *bright, float3 *tmp,
                         cudaStream_t st);
// dst holds a copy of src on entry; its interior pixels are rewritten.
cudaError_t postfx_fxaa(const uint32_t *src, uint32_t *dst, int W, int H, cudaStream_t st);
// sum: 3 floats per pixel.
cudaError_t postfx_accum_add(float *sum, const uint32_t *px, long n, cudaStream_t st);
cudaError_t postfx_accum_resolve(const float *sum, long n, int count, uint32_t *px, cudaStream_t st);

} // namespace rnb
