// Canvas post-processing with reference semantics (src/Renderer.cpp:1353-1470):
// Reinhard tone mapping with gamma, bloom (bright pass, three separable 13-tap box
// blurs, additive blend), FXAA-style edge blending, and the frame accumulation
// buffer. Each output value is formed with the reference's operations in the
// reference's order (this file is compiled with -fmad=false; pow in double, rounded
// once), so results equal the reference's pixel for pixel.
#include <mutex>

#include "common.cuh"
#include "postfx.hpp"

namespace rnb {

namespace {

struct C3 {
	float r, g, b;
};
__device__ __forceinline__ C3 unpack(uint32_t p) {
	return {static_cast<float>((p >> 16) & 0xFFu), static_cast<float>((p >> 8) & 0xFFu),
	        static_cast<float>(p & 0xFFu)};
}
// x86-64 float -> int conversion (cvttss2si): out-of-range and NaN give INT_MIN.
__device__ __forceinline__ int trunc_int(float v) {
	return (v >= -2147483648.0f && v < 2147483648.0f) ? static_cast<int>(v) : static_cast<int>(0x80000000u);
}
__device__ __forceinline__ uint32_t pack(C3 c) {
	const int r = min(255, trunc_int(c.r)), g = min(255, trunc_int(c.g)), b = min(255, trunc_int(c.b));
	return (255u << 24) | ((static_cast<uint32_t>(r) & 0xFFu) << 16) | ((static_cast<uint32_t>(g) & 0xFFu) << 8) |
	       (static_cast<uint32_t>(b) & 0xFFu);
}
__device__ __forceinline__ float pow_f(float x, float y) {
	return static_cast<float>(pow(static_cast<double>(x), static_cast<double>(y)));
}
// (0.299 r + 0.587 g + 0.114 b) / 255
__device__ __forceinline__ float luma(C3 c) { return (0.299f * c.r + 0.587f * c.g + 0.114f * c.b) / 255.0f; }

// toneMap (src/Renderer.cpp:1353-1365)
__global__ void k_tonemap(uint32_t *px, long n, float exposure, float gamma) {
	for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		C3 c = unpack(px[i]);
		c = {c.r / 255.0f * exposure, c.g / 255.0f * exposure, c.b / 255.0f * exposure};
		c = {c.r / (c.r + 1.0f), c.g / (c.g + 1.0f), c.b / (c.b + 1.0f)};
		const float e = 1.0f / gamma;
		c = {pow_f(c.r, e) * 255.0f, pow_f(c.g, e) * 255.0f, pow_f(c.b, e) * 255.0f};
		px[i] = pack(c);
	}
}

// applyBloom's bright pass (src/Renderer.cpp:1393-1403)
__global__ void k_bright(const uint32_t *px, long n, float threshold, float3 *bright) {
	for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const C3 c = unpack(px[i]);
		const float l = luma(c);
		float3 o = make_float3(0.0f, 0.0f, 0.0f);
		if (l > threshold) {
			const float s = l - threshold, d = 1.0f - threshold;
			o = make_float3(c.r * s / d, c.g * s / d, c.b * s / d);
		}
		bright[i] = o;
	}
}

// One 13-tap box blur pass, taps in the reference's order (src/Renderer.cpp:1405-1421).
template <bool kHorizontal>
__global__ void k_box(const float3 *src, float3 *dst, int W, int H) {
	const long n = static_cast<long>(W) * H;
	for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const int x = static_cast<int>(i % W), y = static_cast<int>(i / W);
		float sx = 0.0f, sy = 0.0f, sz = 0.0f;
		int count = 0;
		for (int k = -kPostBlurRadius; k <= kPostBlurRadius; k++) {
			const int ix = kHorizontal ? x + k : x, iy = kHorizontal ? y : y + k;
			if (ix < 0 || ix >= W || iy < 0 || iy >= H)
				continue;
			const float3 v = src[static_cast<long>(iy) * W + ix];
			sx = sx + v.x;
			sy = sy + v.y;
			sz = sz + v.z;
			count++;
		}
		const float cf = static_cast<float>(count);
		dst[i] = make_float3(sx / cf, sy / cf, sz / cf);
	}
}

__global__ void k_bloom_add(uint32_t *px, const float3 *bright, long n, float intensity) {
	for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		C3 c = unpack(px[i]);
		const float3 b = bright[i];
		c = {c.r + b.x * intensity, c.g + b.y * intensity, c.b + b.z * intensity};
		px[i] = pack(c);
	}
}

// applyFXAA (src/Renderer.cpp:1442-1470): reads src, writes interior pixels of dst.
__global__ void k_fxaa(const uint32_t *src, uint32_t *dst, int W, int H) {
	const long n = static_cast<long>(W) * H;
	const float edge = 0.12f;
	for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const int x = static_cast<int>(i % W), y = static_cast<int>(i / W);
		if (x < 1 || y < 1 || x >= W - 1 || y >= H - 1)
			continue;
		const C3 cC = unpack(src[i]), cN = unpack(src[i - W]), cS = unpack(src[i + W]);
		const C3 cW = unpack(src[i - 1]), cE = unpack(src[i + 1]);
		const float lC = luma(cC), lN = luma(cN), lS = luma(cS), lW = luma(cW), lE = luma(cE);
		// std::max / std::min over {lC, lN, lS, lW, lE}
		float mx = lC, mn = lC;
		for (float v : {lN, lS, lW, lE}) {
			if (mx < v)
				mx = v;
			if (v < mn)
				mn = v;
		}
		const float contrast = mx - mn;
		if (contrast < edge)
			continue;
		const C3 avg = {(((cN.r + cS.r) + cW.r) + cE.r) * 0.25f, (((cN.g + cS.g) + cW.g) + cE.g) * 0.25f,
		                (((cN.b + cS.b) + cW.b) + cE.b) * 0.25f};
		const float d = (contrast - edge) * 2.0f;
		const float blend = d < 0.5f ? d : 0.5f; // std::min(0.5f, d)
		// glm::mix(a, b, t) = a * (1 - t) + b * t
		const C3 c = {cC.r * (1.0f - blend) + avg.r * blend, cC.g * (1.0f - blend) + avg.g * blend,
		              cC.b * (1.0f - blend) + avg.b * blend};
		dst[i] = pack(c);
	}
}

// AccumBuffer::add / resolve (src/Renderer.cpp:1373-1391)
__global__ void k_accum_add(float *sum, const uint32_t *px, long n) {
	for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const C3 c = unpack(px[i]);
		sum[3 * i] = sum[3 * i] + c.r;
		sum[3 * i + 1] = sum[3 * i + 1] + c.g;
		sum[3 * i + 2] = sum[3 * i + 2] + c.b;
	}
}
__global__ void k_accum_resolve(const float *sum, long n, float inv, uint32_t *px) {
	for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		px[i] = pack({sum[3 * i] * inv, sum[3 * i + 1] * inv, sum[3 * i + 2] * inv});
}

int grid_for(long n) {
	const long g = (n + 255) / 256;
	return static_cast<int>(g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16);
}

} // namespace

cudaError_t postfx_tonemap(uint32_t *px, long n, float exposure, float gamma, cudaStream_t st) {
	k_tonemap<<<grid_for(n), 256, 0, st>>>(px, n, exposure, gamma);
	return cudaGetLastError();
}

cudaError_t postfx_bloom(uint32_t *px, int W, int H, float threshold, float intensity, float3 *bright, float3 *tmp,
                         cudaStream_t st) {
	const long n = static_cast<long>(W) * H;
	k_bright<<<grid_for(n), 256, 0, st>>>(px, n, threshold, bright);
	for (int pass = 0; pass < 3; pass++) {
		k_box<true><<<grid_for(n), 256, 0, st>>>(bright, tmp, W, H);
		k_box<false><<<grid_for(n), 256, 0, st>>>(tmp, bright, W, H);
	}
	k_bloom_add<<<grid_for(n), 256, 0, st>>>(px, bright, n, intensity);
	return cudaGetLastError();
}

cudaError_t postfx_fxaa(const uint32_t *src, uint32_t *dst, int W, int H, cudaStream_t st) {
	k_fxaa<<<grid_for(static_cast<long>(W) * H), 256, 0, st>>>(src, dst, W, H);
	return cudaGetLastError();
}

cudaError_t postfx_accum_add(float *sum, const uint32_t *px, long n, cudaStream_t st) {
	k_accum_add<<<grid_for(n), 256, 0, st>>>(sum, px, n);
	return cudaGetLastError();
}

cudaError_t postfx_accum_resolve(const float *sum, long n, int count, uint32_t *px, cudaStream_t st) {
	const float inv = count > 0 ? 1.0f / static_cast<float>(count) : 1.0f;
	k_accum_resolve<<<grid_for(n), 256, 0, st>>>(sum, n, inv, px);
	return cudaGetLastError();
}

} // namespace rnb
