// Shared CUDA helpers: error propagation to the C ABI status codes and
// device buffers owned by a scene.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "rednoise/rednoise_pt.h"

namespace rnb {

// Thread-local last error message for rn_pt_last_error().
void set_last_error(const std::string &msg);
const char *get_last_error();

// Testing hook (rn_pt_inject_allocation_failure): true when this device
// allocation is the one chosen to fail.
bool injected_allocation_failure();

// Record a CUDA failure and map it to a status.
rn_status cuda_fail(cudaError_t e, const char *what);

#define RNB_CUDA(call)                                                                                                 \
	do {                                                                                                               \
		cudaError_t e__ = (call);                                                                                      \
		if (e__ != cudaSuccess)                                                                                        \
			return ::rnb::cuda_fail(e__, #call);                                                                       \
	} while (0)

// Debug builds (-DRN_BOUNDS_CHECK, `make debug`) check data-dependent indices
// (tree references, queue slots, sort positions, image pixels) against their
// buffers; a failed check sets the call's status word and skips the access (no
// trap), so the call returns an error. Release builds compile the checks away.
#ifdef RN_BOUNDS_CHECK
constexpr bool kBoundsCheck = true;
#else
constexpr bool kBoundsCheck = false;
#endif

// A device allocation that frees itself.
struct DevBuf {
	void *p = nullptr;
	size_t bytes = 0;
	DevBuf() = default;
	DevBuf(const DevBuf &) = delete;
	DevBuf &operator=(const DevBuf &) = delete;
	~DevBuf() { release(); }
	void release() {
		if (p)
			cudaFree(p);
		p = nullptr;
		bytes = 0;
	}
	// Grow-only (re)allocation; contents are not preserved.
	cudaError_t ensure(size_t n) {
		if (n <= bytes)
			return cudaSuccess;
		release();
		if (injected_allocation_failure())
			return cudaErrorMemoryAllocation;
		cudaError_t e = cudaMalloc(&p, n);
		if (e == cudaSuccess)
			bytes = n;
		else
			p = nullptr;
		return e;
	}
	template <typename T> T *as() const { return static_cast<T *>(p); }
};

inline int ceil_div(long a, long b) { return static_cast<int>((a + b - 1) / b); }

} // namespace rnb
