// rn_pt_render_static: a physical-mode render that allocates no memory.
//
// Some callers cannot call cudaMalloc while they render: code that runs under
// another framework's memory manager, real-time loops that must not touch the
// allocator, or hosts that hand the library a fixed memory budget. For them this
// entry point runs the megakernel with its scratch -- the per-pixel sample sums
// and the persistent warps' work counter -- in a fixed array compiled into this
// library, and writes the mean radiance to the caller's device buffer. The scene
// must already be prepared (rn_pt_scene_prepare), since preparing allocates; a
// traversal error lands in the scene's status word, which the scene's next
// synchronising call reports, as for rn_pt_render with device pointers.
//
// The array is kStaticScratchBytes long and lives on every GPU that loads the
// library until the process exits. It holds at most kStaticMaxPixels pixels; larger
// images are rejected. All calls share it and it keeps the previous call's
// contents, so each call clears the parts that must start at zero; calls whose GPU
// work overlaps (two streams, two threads) race on it and must be serialised by
// the caller. The output must be device (or managed) memory of the scene's GPU:
// the pointer is checked with cudaPointerGetAttributes, which allocates nothing,
// before any GPU work, so a host buffer is refused instead of being written by a
// kernel. The array's device address is looked up once per device and kept for
// the life of the process; cudaDeviceReset unloads the module that holds the
// array, so calling this entry point after a reset of the device is unsupported.
#include <mutex>

#include "pt_kernels.hpp"
#include "render_impl.hpp"
#include "scene_impl.hpp"

namespace rnb {

constexpr long kStaticMaxPixels = RN_PT_STATIC_MAX_PIXELS;
constexpr size_t kStaticHeaderBytes = 256; // work counter, padded to keep the sums 256-byte aligned
constexpr size_t kStaticScratchBytes = kStaticHeaderBytes + static_cast<size_t>(kStaticMaxPixels) * 3 * sizeof(float);

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
void *g_static_ptr[kMaxDevices] = {};

// Device address of the array for the current device. The first call on each
// device resolves it (cudaGetSymbolAddress, with that device current) and keeps
// it; make that first call before any stream capture on the device.
rn_status static_scratch(void **out) {
	int dev = 0;
	RNB_CUDA(cudaGetDevice(&dev));
	if (dev < 0 || dev >= kMaxDevices) {
		set_last_error("rn_pt_render_static: device ordinal out of range");
		return RN_ERR_UNSUPPORTED;
	}
	std::lock_guard<std::mutex> lock(g_static_mu);
	if (!g_static_ptr[dev]) {
		void *p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
		if (e != cudaSuccess || !p)
			return cuda_fail(e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress(g_static_scratch)");
		g_static_ptr[dev] = p;
	}
	*out = g_static_ptr[dev];
	return RN_OK;
}

} // namespace

} // namespace rnb

using namespace rnb;

extern "C" {

rn_status rn_pt_render_static(rn_scene *scene, const rn_pt_camera *camera, const rn_pt_settings *settings,
                              unsigned flags, void *stream, float *rgb) {
	if (!scene || !camera || !settings || !rgb) {
		set_last_error("rn_pt_render_static: NULL argument");
		return RN_ERR_INVALID_ARGUMENT;
	}
	bool prepared;
	{
		std::lock_guard<std::mutex> lock(scene->mu); // prepare_scene sets the flag under this lock
		prepared = scene->prepared;
	}
	if (!prepared) {
		set_last_error("rn_pt_render_static: prepare the scene first (rn_pt_scene_prepare allocates)");
		return RN_ERR_INVALID_ARGUMENT;
	}
	const long npix = static_cast<long>(camera->width) * camera->height;
	if (camera->width <= 0 || camera->height <= 0 || npix > kStaticMaxPixels) {
		set_last_error("rn_pt_render_static: image must have between 1 and 262144 pixels (512 x 512), the size of "
		               "the library's fixed scratch");
		return RN_ERR_CAPACITY;
	}
	PhysScene ps;
	PhysCamera pc;
	PhysSettings pst;
	rn_status r = make_phys_inputs(scene, camera, settings, flags, ps, pc, pst);
	if (r != RN_OK)
		return r;
	int dev = -1;
	RNB_CUDA(cudaGetDevice(&dev));
	if (dev != scene->device) {
		set_last_error("rn_pt_render_static: make the scene's device current first");
		return RN_ERR_INVALID_ARGUMENT;
	}
	// The output must be memory a kernel on this device may write: a host buffer
	// (pageable or pinned) is refused here, before any GPU work.
	cudaPointerAttributes pa{};
	const cudaError_t pe = cudaPointerGetAttributes(&pa, rgb);
	if (pe != cudaSuccess) {
		(void)cudaGetLastError(); // an unknown pointer also sets the thread's last CUDA error; clear it
		set_last_error("rn_pt_render_static: rgb is not a CUDA device pointer");
		return RN_ERR_INVALID_ARGUMENT;
	}
	if (!((pa.type == cudaMemoryTypeDevice && pa.device == dev) || pa.type == cudaMemoryTypeManaged)) {
		set_last_error("rn_pt_render_static: rgb must be device memory of the scene's GPU (or managed memory); "
		               "host buffers are not accepted");
		return RN_ERR_INVALID_ARGUMENT;
	}
	void *base = nullptr;
	r = static_scratch(&base);
	if (r != RN_OK)
		return r;
	unsigned char *b = static_cast<unsigned char *>(base);
	unsigned *counter = reinterpret_cast<unsigned *>(b);
	float *accum = reinterpret_cast<float *>(b + kStaticHeaderBytes);
	const size_t bytes = static_cast<size_t>(npix) * 3 * sizeof(float);
	cudaStream_t cs = stream ? static_cast<cudaStream_t>(stream) : scene->stream;
	RNB_CUDA(cudaMemsetAsync(b, 0, kStaticHeaderBytes, cs));
	RNB_CUDA(cudaMemsetAsync(accum, 0, bytes, cs));
	RNB_CUDA(launch_megakernel(ps, pc, pst, accum, counter, scene->d_status.as<int>(), cs));
	RNB_CUDA(launch_resolve(accum, rgb, npix * 3, pst.spp > 0 ? 1.0f / static_cast<float>(pst.spp) : 0.0f, cs));
	return RN_OK;
}

} // extern "C"
