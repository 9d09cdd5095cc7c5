// Read-bandwidth probe for the roofline denominators of the traversal kernels.
//
// The traversal's working set (the 4-wide tree and the triangles) is served from
// L1 and L2, not from HBM, so its roofline needs the bandwidth of an L2-resident
// read on this GPU. A persistent grid (eight 256-thread blocks per SM) reads the
// caller's buffer `passes` times per launch with 16-byte loads in a grid-stride
// loop (enough passes make a launch long against its launch overhead); with
// l2_only the loads bypass L1 (ld.global.cg), so a buffer well under the L2's
// size measures the L2's read bandwidth, and one far above it measures HBM.
#include "scene_impl.hpp"

namespace rnb {
namespace {

// Destination of the probe's sum, which is only written when it takes a value no
// real input produces; the condition keeps the compiler from dropping the loads.
__device__ float g_probe_sink;

template <bool kL2Only>
__global__ void __launch_bounds__(256) k_probe_read(const float4 *__restrict__ p, size_t n4, int passes) {
	float acc = 0.0f;
	const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
	for (int pass = 0; pass < passes; pass++) {
		for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n4; i += stride) {
			const float4 v = kL2Only ? __ldcg(p + i) : __ldg(p + i);
			acc += (v.x + v.y) + (v.z + v.w);
		}
	}
	if (acc == -1.2345678e30f)
		g_probe_sink = acc;
}

} // namespace
} // namespace rnb

using namespace rnb;

extern "C" {

rn_status rn_pt_probe_read(const void *buf, size_t bytes, int passes, int launches, int l2_only, void *stream,
                           float *ms) {
	if (!buf || !ms || launches < 1 || passes < 1 || bytes < 16 || (reinterpret_cast<uintptr_t>(buf) & 15) != 0) {
		set_last_error("rn_pt_probe_read: need a 16-byte aligned device buffer of at least 16 bytes, passes >= 1, "
		               "launches >= 1 and ms");
		return RN_ERR_INVALID_ARGUMENT;
	}
	int dev = 0, sms = 148;
	RNB_CUDA(cudaGetDevice(&dev));
	RNB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
	cudaStream_t cs = static_cast<cudaStream_t>(stream);
	const size_t n4 = bytes / 16;
	const float4 *p = static_cast<const float4 *>(buf);
	cudaEvent_t a = nullptr, b = nullptr;
	RNB_CUDA(cudaEventCreate(&a));
	cudaError_t e = cudaEventCreate(&b);
	if (e == cudaSuccess) {
		// one untimed launch brings an L2-sized buffer into L2
		if (l2_only)
			k_probe_read<true><<<sms * 8, 256, 0, cs>>>(p, n4, passes);
		else
			k_probe_read<false><<<sms * 8, 256, 0, cs>>>(p, n4, passes);
		e = cudaEventRecord(a, cs);
		for (int i = 0; e == cudaSuccess && i < launches; i++) {
			if (l2_only)
				k_probe_read<true><<<sms * 8, 256, 0, cs>>>(p, n4, passes);
			else
				k_probe_read<false><<<sms * 8, 256, 0, cs>>>(p, n4, passes);
			e = cudaGetLastError();
		}
		if (e == cudaSuccess)
			e = cudaEventRecord(b, cs);
		if (e == cudaSuccess)
			e = cudaEventSynchronize(b);
		if (e == cudaSuccess)
			e = cudaEventElapsedTime(ms, a, b);
	}
	cudaEventDestroy(a);
	if (b)
		cudaEventDestroy(b);
	if (e != cudaSuccess)
		return cuda_fail(e, "rn_pt_probe_read");
	return RN_OK;
}

} // extern "C"
