// TEST INFRASTRUCTURE ONLY -- counter-based RNG of the oracle.
//
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11), restated from the published description: ten rounds of
// two 32x32->64 multiplies with the Weyl key schedule. The physical-mode
// integrator keys it by (seed) and counts (pixel, sample, bounce, stream), so
// the GPU and this oracle draw identical uniforms for the same path.
#pragma once

#include <cstdint>

namespace orc {

struct U4 {
	uint32_t x, y, z, w;
};

inline U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
	const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
	for (int r = 0; r < 10; r++) {
		const uint64_t p0 = static_cast<uint64_t>(M0) * c.x;
		const uint64_t p1 = static_cast<uint64_t>(M1) * c.z;
		const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
		const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
		c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
		k0 += W0;
		k1 += W1;
	}
	return c;
}

// 24-bit uniform in [0, 1): exact in float and double alike.
inline float u01(uint32_t x) { return static_cast<float>(x >> 8) * (1.0f / 16777216.0f); }

} // namespace orc
