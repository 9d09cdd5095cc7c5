// The plain GPU megakernel: one thread traces every sample of one pixel through
// closest hit, shading, shadow ray and continuation in a single kernel.
// Persistent warps fetch 32-pixel batches from a global counter. Samples are
// summed in sample order onto the incoming accumulator, so a render split into
// several calls with sample offsets equals a single call bit for bit.
#include "pt_kernels.hpp"

namespace rnb {

template <int kOrder>
__global__ void __launch_bounds__(128) k_megakernel(PhysScene sc, PhysCamera cam, PhysSettings st,
                                                    float *__restrict__ accum, unsigned *__restrict__ counter,
                                                    int n_pixels, int *status) {
	int err = 0;
	const int lane = threadIdx.x & 31;
	for (;;) {
		int base = 0;
		if (lane == 0)
			base = static_cast<int>(atomicAdd(counter, 32u));
		base = __shfl_sync(0xffffffffu, base, 0);
		if (base >= n_pixels)
			break;
		const int pix = base + lane;
		if (pix < n_pixels) {
			F3 sum = f3(accum[3 * pix], accum[3 * pix + 1], accum[3 * pix + 2]);
			for (int s = 0; s < st.spp; s++) {
				PathState ps = camera_path(cam, st, static_cast<uint32_t>(pix), st.sample_offset + static_cast<uint32_t>(s));
				for (;;) {
					const RayPre r = make_ray(ps.o.x, ps.o.y, ps.o.z, ps.d.x, ps.d.y, ps.d.z);
					const HitRec h = trace_closest_best<kOrder>(sc.sv, r, ps.ignore, err);
					ShadowReq sr;
					const bool alive = shade_vertex(sc, st, ps, h, sr);
					if (sr.valid) {
						const RayPre rs = make_ray(sr.o.x, sr.o.y, sr.o.z, sr.d.x, sr.d.y, sr.d.z);
						if (!trace_any_best(sc.sv, rs, sr.tmax, sr.ignore, err))
							ps.L = ps.L + sr.contrib;
					}
					if (!alive)
						break;
				}
				sum = sum + ps.L;
			}
			accum[3 * pix] = sum.x;
			accum[3 * pix + 1] = sum.y;
			accum[3 * pix + 2] = sum.z;
		}
	}
	if (err)
		atomicOr(status, 1);
}

// Counters: [0] samples, [1] closest queries, [2] any-hit queries, [3] closest box
// tests, [4] closest triangle tests, [5] any-hit box tests, [6] any-hit triangle tests.
__global__ void __launch_bounds__(128) k_count(PhysScene sc, PhysCamera cam, PhysSettings st, int n_pixels,
                                               unsigned long long *__restrict__ out, int *status) {
	int err = 0;
	unsigned long long c[7] = {0, 0, 0, 0, 0, 0, 0};
	for (int pix = blockIdx.x * blockDim.x + threadIdx.x; pix < n_pixels; pix += gridDim.x * blockDim.x) {
		for (int s = 0; s < st.spp; s++) {
			PathState ps = camera_path(cam, st, static_cast<uint32_t>(pix), st.sample_offset + static_cast<uint32_t>(s));
			c[0]++;
			for (;;) {
				const RayPre r = make_ray(ps.o.x, ps.o.y, ps.o.z, ps.d.x, ps.d.y, ps.d.z);
				HitRec h;
				c[1]++;
				count_reference_query<false>(sc.sv, r, ps.ignore, 0.0f, h, c[3], c[4], err);
				ShadowReq sr;
				const bool alive = shade_vertex(sc, st, ps, h, sr);
				if (sr.valid) {
					const RayPre rs = make_ray(sr.o.x, sr.o.y, sr.o.z, sr.d.x, sr.d.y, sr.d.z);
					HitRec dummy;
					c[2]++;
					if (!count_reference_query<true>(sc.sv, rs, sr.ignore, sr.tmax, dummy, c[5], c[6], err))
						ps.L = ps.L + sr.contrib;
				}
				if (!alive)
					break;
			}
		}
	}
	for (int k = 0; k < 7; k++) {
		unsigned long long v = c[k];
		for (int o = 16; o > 0; o >>= 1)
			v += __shfl_down_sync(0xffffffffu, v, o);
		if ((threadIdx.x & 31) == 0 && v)
			atomicAdd(out + k, v);
	}
	if (err)
		atomicOr(status, 1);
}

cudaError_t launch_count(const PhysScene &sc, const PhysCamera &cam, const PhysSettings &st, unsigned long long *out,
                         int *status, cudaStream_t stream) {
	const int n = cam.width * cam.height;
	cudaError_t e = cudaMemsetAsync(out, 0, 7 * sizeof(unsigned long long), stream);
	if (e != cudaSuccess || n <= 0)
		return e;
	const int blocks = (n + 127) / 128 < 148 * 16 ? (n + 127) / 128 : 148 * 16;
	k_count<<<blocks, 128, 0, stream>>>(sc, cam, st, n, out, status);
	return cudaGetLastError();
}

__global__ void k_resolve(const float *__restrict__ accum, float *__restrict__ mean, long n, float inv) {
	for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
	     i += static_cast<long>(gridDim.x) * blockDim.x)
		mean[i] = accum[i] * inv;
}

cudaError_t launch_resolve(const float *accum, float *mean, long n_floats, float inv_spp, cudaStream_t stream) {
	if (n_floats <= 0)
		return cudaSuccess;
	const int blocks = static_cast<int>((n_floats + 255) / 256 < 148 * 32 ? (n_floats + 255) / 256 : 148 * 32);
	k_resolve<<<blocks, 256, 0, stream>>>(accum, mean, n_floats, inv_spp);
	return cudaGetLastError();
}

cudaError_t launch_megakernel(const PhysScene &sc, const PhysCamera &cam, const PhysSettings &st, float *accum,
                              unsigned *counter, int *status, cudaStream_t stream) {
	const int n = cam.width * cam.height;
	if (n <= 0 || st.spp <= 0)
		return cudaSuccess;
	cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned), stream);
	if (e != cudaSuccess)
		return e;
	int dev = 0, sms = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	int per_sm = 0;
	if (st.order == kOrderNearest)
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_megakernel<kOrderNearest>, 128, 0);
	else
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_megakernel<kOrderReference>, 128, 0);
	if (per_sm < 1)
		per_sm = 1;
	int blocks = sms * per_sm;
	const int needed = (n + 127) / 128;
	if (blocks > needed)
		blocks = needed;
	if (st.order == kOrderNearest)
		k_megakernel<kOrderNearest><<<blocks, 128, 0, stream>>>(sc, cam, st, accum, counter, n, status);
	else
		k_megakernel<kOrderReference><<<blocks, 128, 0, stream>>>(sc, cam, st, accum, counter, n, status);
	return cudaGetLastError();
}

} // namespace rnb
