// Counter-based random numbers for the physical-mode integrators.
//
// Philox-4x32-10 (Salmon et al., SC'11): ten rounds of two 32x32->64-bit
// multiplies with the Weyl key schedule. A path draws its uniforms from the
// counter (pixel, sample, block, 0) under the key (seed), so any kernel -- the
// megakernel, the wavefront stages, the adjoint replay -- regenerates the same
// numbers for the same path without storing them.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rnb {

struct U4 {
	uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
	const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#ifdef __CUDACC__
#pragma unroll
#endif
	for (int r = 0; r < 10; r++) {
#ifdef __CUDA_ARCH__
		const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
		const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
#else
		const uint64_t p0 = static_cast<uint64_t>(M0) * c.x, p1 = static_cast<uint64_t>(M1) * c.z;
		const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
		const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
#endif
		c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
		k0 += W0;
		k1 += W1;
	}
	return c;
}

// 24-bit uniform in [0, 1), exactly representable in float.
__host__ __device__ __forceinline__ float u01(uint32_t x) { return static_cast<float>(x >> 8) * (1.0f / 16777216.0f); }

// Counter blocks of one path: block 0 = camera jitter, 2 + 2*b and 3 + 2*b = vertex b.
__host__ __device__ __forceinline__ U4 path_rand(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t block) {
	return philox4x32_10(U4{pixel, sample, block, 0u}, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
}

} // namespace rnb
