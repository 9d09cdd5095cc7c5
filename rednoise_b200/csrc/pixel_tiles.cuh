// Pixel visiting order for the wavefront's camera rays: 8 x 4 pixel tiles in
// row-major tile order (one warp per tile), then the pixels the full tiles leave
// over (the right strip row by row, then the bottom strip). A warp's camera rays
// then start from a compact patch of the image instead of a 32-pixel row strip.
// Only the order in which pixels are taken changes; each pixel keeps its own
// random stream and output location.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define RNB_TILE_FN __host__ __device__ __forceinline__
#else
#define RNB_TILE_FN inline // host-only builds (the host tests)
#endif

namespace rnb {

// Position of row-major pixel p of a w x h image in tile order (a bijection on [0, w h)).
RNB_TILE_FN uint32_t tile_order(uint32_t p, uint32_t w, uint32_t h) {
	const uint32_t x = p % w, y = p / w;
	const uint32_t w8 = w - w % 8, h4 = h - h % 4;
	if (x < w8 && y < h4)
		return ((y / 4) * (w8 / 8) + x / 8) * 32 + (y % 4) * 8 + x % 8;
	if (y < h4)
		return w8 * h4 + y * (w - w8) + (x - w8);
	return w8 * h4 + h4 * (w - w8) + (y - h4) * w + x;
}

} // namespace rnb
