// Pixel visiting order for the wavefront's camera rays: 8 x 4 pixel tiles in
// row-major tile order (one warp per tile), then the pixels the full tiles leave
// over (the right strip row by row, then the bottom strip). A warp's camera rays
// then start from a compact patch of the image instead of a 32-pixel row strip.
// Only the order in which pixels are taken changes; each pixel keeps its own
// random stream and output location. tile_pixel is the inverse map.
#pragma once

#include <stdint.h>

namespace rnb {

// Position of row-major pixel p of a w x h image in tile order (a bijection on [0, w h)).
__device__ __forceinline__ uint32_t tile_order(uint32_t p, uint32_t w, uint32_t h) {
	const uint32_t x = p % w, y = p / w;
	const uint32_t w8 = w - w % 8, h4 = h - h % 4;
	if (x < w8 && y < h4)
		return ((y / 4) * (w8 / 8) + x / 8) * 32 + (y % 4) * 8 + x % 8;
	if (y < h4)
		return w8 * h4 + y * (w - w8) + (x - w8);
	return w8 * h4 + h4 * (w - w8) + (y - h4) * w + x;
}

// The inverse: the row-major pixel at position t of the tile order.
__device__ __forceinline__ uint32_t tile_pixel(uint32_t t, uint32_t w, uint32_t h) {
	const uint32_t w8 = w - w % 8, h4 = h - h % 4;
	const uint32_t full = w8 * h4, strip = h4 * (w - w8);
	if (t < full) {
		const uint32_t tile = t / 32, r = t % 32;
		const uint32_t tx = tile % (w8 / 8), ty = tile / (w8 / 8);
		return (ty * 4 + r / 8) * w + tx * 8 + r % 8;
	}
	if (t < full + strip) {
		const uint32_t u = t - full;
		return (u / (w - w8)) * w + w8 + u % (w - w8);
	}
	const uint32_t u = t - full - strip;
	return (h4 + u / w) * w + u % w;
}

} // namespace rnb
