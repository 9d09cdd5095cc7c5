// C ABI of the canvas post-processing (toneMap, applyBloom, applyFXAA, AccumBuffer).
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "postfx.hpp"
#include "rednoise/rednoise_pt.h"

using namespace rnb;

namespace {

// One scratch buffer per process for host-array calls and the filters' work
// arrays; calls are serialised on it.
std::mutex g_mu;
DevBuf g_scratch;
int g_device = -1;

rn_status check_canvas(const void *p, int w, int h, const char *what) {
	if (!p || w <= 0 || h <= 0 || static_cast<long>(w) * h > (1L << 28)) {
		set_last_error(std::string(what) + ": need a canvas pointer and 1 <= width*height <= 2^28");
		return RN_ERR_INVALID_ARGUMENT;
	}
	return RN_OK;
}

// Scratch of at least `bytes`, on the current device.
rn_status scratch(size_t bytes, char **out) {
	int dev = 0;
	RNB_CUDA(cudaGetDevice(&dev));
	if (dev != g_device) {
		g_scratch.release();
		g_device = dev;
	}
	RNB_CUDA(g_scratch.ensure(bytes));
	*out = g_scratch.as<char>();
	return RN_OK;
}

inline size_t a256(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }

// Runs fn on a device canvas: the caller's (device mode) or a scratch copy of the
// caller's host canvas, copied back after.
template <typename Fn>
rn_status on_canvas(uint32_t *argb, long n, size_t extra, unsigned flags, void *stream, const char *what, Fn fn) {
	const bool dev = (flags & RN_PT_DEVICE_POINTERS) != 0;
	cudaStream_t cs = static_cast<cudaStream_t>(stream);
	std::lock_guard<std::mutex> lock(g_mu);
	char *base = nullptr;
	rn_status r = scratch((dev ? 0 : a256(static_cast<size_t>(n) * 4)) + extra + 256, &base);
	if (r != RN_OK)
		return r;
	uint32_t *px = dev ? argb : reinterpret_cast<uint32_t *>(base);
	char *work = base + (dev ? 0 : a256(static_cast<size_t>(n) * 4));
	if (!dev)
		RNB_CUDA(cudaMemcpyAsync(px, argb, static_cast<size_t>(n) * 4, cudaMemcpyHostToDevice, cs));
	r = fn(px, work);
	if (r != RN_OK)
		return r;
	if (!dev)
		RNB_CUDA(cudaMemcpyAsync(argb, px, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToHost, cs));
	// the scratch is shared: finish before releasing it
	RNB_CUDA(cudaStreamSynchronize(cs));
	(void)what;
	return RN_OK;
}

} // namespace

extern "C" {

rn_status rn_pt_tonemap(uint32_t *argb, int width, int height, float exposure, float gamma, unsigned flags,
                        void *stream) {
	rn_status r = check_canvas(argb, width, height, "rn_pt_tonemap");
	if (r != RN_OK)
		return r;
	const long n = static_cast<long>(width) * height;
	return on_canvas(argb, n, 0, flags, stream, "rn_pt_tonemap", [&](uint32_t *px, char *) -> rn_status {
		RNB_CUDA(postfx_tonemap(px, n, exposure, gamma, static_cast<cudaStream_t>(stream)));
		return RN_OK;
	});
}

rn_status rn_pt_bloom(uint32_t *argb, int width, int height, float threshold, float intensity, unsigned flags,
                      void *stream) {
	rn_status r = check_canvas(argb, width, height, "rn_pt_bloom");
	if (r != RN_OK)
		return r;
	const long n = static_cast<long>(width) * height;
	const size_t f3 = a256(static_cast<size_t>(n) * sizeof(float3));
	return on_canvas(argb, n, 2 * f3, flags, stream, "rn_pt_bloom", [&](uint32_t *px, char *work) -> rn_status {
		RNB_CUDA(postfx_bloom(px, width, height, threshold, intensity, reinterpret_cast<float3 *>(work),
		                      reinterpret_cast<float3 *>(work + f3), static_cast<cudaStream_t>(stream)));
		return RN_OK;
	});
}

rn_status rn_pt_fxaa(uint32_t *argb, int width, int height, unsigned flags, void *stream) {
	rn_status r = check_canvas(argb, width, height, "rn_pt_fxaa");
	if (r != RN_OK)
		return r;
	const long n = static_cast<long>(width) * height;
	return on_canvas(argb, n, a256(static_cast<size_t>(n) * 4), flags, stream, "rn_pt_fxaa",
	                 [&](uint32_t *px, char *work) -> rn_status {
		                 uint32_t *src = reinterpret_cast<uint32_t *>(work);
		                 cudaStream_t cs = static_cast<cudaStream_t>(stream);
		                 RNB_CUDA(cudaMemcpyAsync(src, px, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToDevice, cs));
		                 RNB_CUDA(postfx_fxaa(src, px, width, height, cs));
		                 return RN_OK;
	                 });
}

rn_status rn_pt_accum_add(float *sum, const uint32_t *argb, int width, int height, unsigned flags, void *stream) {
	rn_status r = check_canvas(argb, width, height, "rn_pt_accum_add");
	if (r != RN_OK || !sum) {
		if (r == RN_OK)
			set_last_error("rn_pt_accum_add: NULL sum");
		return r == RN_OK ? RN_ERR_INVALID_ARGUMENT : r;
	}
	const long n = static_cast<long>(width) * height;
	cudaStream_t cs = static_cast<cudaStream_t>(stream);
	if (flags & RN_PT_DEVICE_POINTERS) {
		RNB_CUDA(postfx_accum_add(sum, argb, n, cs));
		return RN_OK;
	}
	std::lock_guard<std::mutex> lock(g_mu);
	char *base = nullptr;
	const size_t sb = a256(static_cast<size_t>(n) * 12);
	r = scratch(sb + a256(static_cast<size_t>(n) * 4), &base);
	if (r != RN_OK)
		return r;
	float *d_sum = reinterpret_cast<float *>(base);
	uint32_t *d_px = reinterpret_cast<uint32_t *>(base + sb);
	RNB_CUDA(cudaMemcpyAsync(d_sum, sum, static_cast<size_t>(n) * 12, cudaMemcpyHostToDevice, cs));
	RNB_CUDA(cudaMemcpyAsync(d_px, argb, static_cast<size_t>(n) * 4, cudaMemcpyHostToDevice, cs));
	RNB_CUDA(postfx_accum_add(d_sum, d_px, n, cs));
	RNB_CUDA(cudaMemcpyAsync(sum, d_sum, static_cast<size_t>(n) * 12, cudaMemcpyDeviceToHost, cs));
	RNB_CUDA(cudaStreamSynchronize(cs));
	return RN_OK;
}

rn_status rn_pt_accum_resolve(const float *sum, int count, uint32_t *argb, int width, int height, unsigned flags,
                              void *stream) {
	rn_status r = check_canvas(argb, width, height, "rn_pt_accum_resolve");
	if (r != RN_OK || !sum) {
		if (r == RN_OK)
			set_last_error("rn_pt_accum_resolve: NULL sum");
		return r == RN_OK ? RN_ERR_INVALID_ARGUMENT : r;
	}
	const long n = static_cast<long>(width) * height;
	cudaStream_t cs = static_cast<cudaStream_t>(stream);
	if (flags & RN_PT_DEVICE_POINTERS) {
		RNB_CUDA(postfx_accum_resolve(sum, n, count, argb, cs));
		return RN_OK;
	}
	std::lock_guard<std::mutex> lock(g_mu);
	char *base = nullptr;
	const size_t sb = a256(static_cast<size_t>(n) * 12);
	r = scratch(sb + a256(static_cast<size_t>(n) * 4), &base);
	if (r != RN_OK)
		return r;
	float *d_sum = reinterpret_cast<float *>(base);
	uint32_t *d_px = reinterpret_cast<uint32_t *>(base + sb);
	RNB_CUDA(cudaMemcpyAsync(d_sum, sum, static_cast<size_t>(n) * 12, cudaMemcpyHostToDevice, cs));
	RNB_CUDA(postfx_accum_resolve(d_sum, n, count, d_px, cs));
	RNB_CUDA(cudaMemcpyAsync(argb, d_px, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToHost, cs));
	RNB_CUDA(cudaStreamSynchronize(cs));
	return RN_OK;
}

} // extern "C"
