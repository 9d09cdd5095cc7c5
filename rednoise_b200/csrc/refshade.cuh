// Shared device code of the reference-semantics renderers (path tracer, Whitted
// ray tracer, photon mapper): glm-order vector arithmetic, libm-equivalent
// transcendental functions, std::mt19937 and libstdc++'s uniform_real_distribution
// mapping, Ken Perlin's improved noise, the reference's visibility patterns,
// direct lighting, cosine-hemisphere sampling, sky and surface colour.
//
// Include only from translation units compiled with -fmad=false: the arithmetic
// must be evaluated as separately rounded IEEE operations in source order to
// reproduce the reference's non-FMA x86-64 build.
#pragma once

#include <cstdint>

#include "refmode.hpp"
#include "scene_impl.hpp"

namespace rnb {
namespace {


struct V3 {
	float x, y, z;
};
__device__ __forceinline__ V3 mk(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
// glm dot: tmp = a*b; (tmp.x + tmp.y) + tmp.z
__device__ __forceinline__ float dot(V3 a, V3 b) {
	const float x = a.x * b.x, y = a.y * b.y, z = a.z * b.z;
	return (x + y) + z;
}
__device__ __forceinline__ V3 cross(V3 x, V3 y) {
	return {x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y};
}
__device__ __forceinline__ float length(V3 v) { return sqrtf(dot(v, v)); }
// glm normalize: v * inversesqrt(dot(v, v)), inversesqrt = 1 / sqrt(x)
__device__ __forceinline__ V3 normalize(V3 v) { return v * (1.0f / sqrtf(dot(v, v))); }
// glm reflect: I - N * dot(N, I) * 2
__device__ __forceinline__ V3 reflect(V3 I, V3 N) { return I - (N * dot(N, I)) * 2.0f; }
// glm refract
__device__ __forceinline__ V3 refract(V3 I, V3 N, float eta) {
	const float dv = dot(N, I);
	const float k = 1.0f - eta * eta * (1.0f - dv * dv);
	if (k >= 0.0f)
		return eta * I - (eta * dv + sqrtf(k)) * N;
	return mk(0.0f, 0.0f, 0.0f);
}
// glm mix(x, y, a) = x * (1 - a) + y * a
__device__ __forceinline__ V3 mix(V3 x, V3 y, float a) { return x * (1.0f - a) + y * a; }
__device__ __forceinline__ float gmin(float x, float y) { return (y < x) ? y : x; }
__device__ __forceinline__ V3 vmin(V3 a, V3 b) { return {gmin(a.x, b.x), gmin(a.y, b.y), gmin(a.z, b.z)}; }
// std::max(a, b) = (a < b) ? b : a
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ V3 face_viewer(V3 n, V3 d) { return dot(n, d) > 0.0f ? -n : n; }

// libm-equivalent single-precision transcendental functions (see file header).
__device__ __forceinline__ float lm_cos(float x) { return static_cast<float>(cos(static_cast<double>(x))); }
__device__ __forceinline__ float lm_sin(float x) { return static_cast<float>(sin(static_cast<double>(x))); }
__device__ __forceinline__ float lm_exp(float x) { return static_cast<float>(exp(static_cast<double>(x))); }
__device__ __forceinline__ float lm_pow(float x, float y) {
	return static_cast<float>(pow(static_cast<double>(x), static_cast<double>(y)));
}

// ---- std::mt19937 (Matsumoto & Nishimura 1998), 32-bit, default parameters ----
struct MT {
	uint32_t s[624];
	int i;
	__device__ void seed(uint32_t v) {
		s[0] = v;
		for (int k = 1; k < 624; k++)
			s[k] = 1812433253u * (s[k - 1] ^ (s[k - 1] >> 30)) + static_cast<uint32_t>(k);
		i = 624;
	}
	__device__ void twist() {
		for (int k = 0; k < 624; k++) {
			const uint32_t y = (s[k] & 0x80000000u) | (s[k + 1 < 624 ? k + 1 : 0] & 0x7fffffffu);
			const int m = k + 397 < 624 ? k + 397 : k + 397 - 624;
			s[k] = s[m] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
		}
		i = 0;
	}
	__device__ uint32_t next() {
		if (i >= 624)
			twist();
		uint32_t y = s[i++];
		y ^= y >> 11;
		y ^= (y << 7) & 0x9d2c5680u;
		y ^= (y << 15) & 0xefc60000u;
		y ^= y >> 18;
		return y;
	}
	// uniform_real_distribution<float>(a, b): canonical * (b - a) + a with
	// canonical = float(x) / 2^32, clamped below 1 (libstdc++ generate_canonical).
	__device__ float uniform(float a, float b) {
		float c = __uint2float_rn(next()) / 4294967296.0f;
		if (c >= 1.0f)
			c = 0.99999994f;
		return c * (b - a) + a;
	}
};

// std::mt19937 for streams that are freshly seeded per pixel: the first 227
// outputs of a seeded state's first twist depend only on the seed sequence
// s[i], s[i + 1] and s[i + 397], which two running cursors over the seeding
// recurrence provide in registers -- no 2.5 KB state is written or read. From
// output 227 on (where the twist needs words it has already replaced) the full
// state is built as MT does, so every output equals MT's.
struct MtFresh {
	uint32_t seed_v, a, b; // seed value; cursors: a = s[i], b = s[i + 397]
	int i;                 // outputs drawn so far
	bool full;
	MT mt;
	__device__ void seed(uint32_t v) {
		seed_v = v;
		a = v;
		b = v;
		for (int k = 1; k <= 397; k++)
			b = 1812433253u * (b ^ (b >> 30)) + static_cast<uint32_t>(k);
		i = 0;
		full = false;
	}
	__device__ uint32_t next() {
		if (!full) {
			if (i < 227) {
				const uint32_t a1 = 1812433253u * (a ^ (a >> 30)) + static_cast<uint32_t>(i + 1);
				const uint32_t y0 = (a & 0x80000000u) | (a1 & 0x7fffffffu);
				uint32_t y = b ^ (y0 >> 1) ^ ((y0 & 1u) ? 0x9908b0dfu : 0u);
				a = a1;
				b = 1812433253u * (b ^ (b >> 30)) + static_cast<uint32_t>(i + 398);
				i++;
				y ^= y >> 11;
				y ^= (y << 7) & 0x9d2c5680u;
				y ^= (y << 15) & 0xefc60000u;
				y ^= y >> 18;
				return y;
			}
			mt.seed(seed_v);
			mt.twist();
			mt.i = 227;
			full = true;
		}
		return mt.next();
	}
	__device__ float uniform(float lo, float hi) {
		float c = __uint2float_rn(next()) / 4294967296.0f;
		if (c >= 1.0f)
			c = 0.99999994f;
		return c * (hi - lo) + lo;
	}
};

// ---- Ken Perlin's improved noise (2002), as the reference's procedural colour uses ----
__constant__ uint8_t kPerm[256] = {
    151, 160, 137, 91,  90,  15,  131, 13,  201, 95,  96,  53,  194, 233, 7,   225, 140, 36,  103, 30,  69,  142,
    8,   99,  37,  240, 21,  10,  23,  190, 6,   148, 247, 120, 234, 75,  0,   26,  197, 62,  94,  252, 219, 203,
    117, 35,  11,  32,  57,  177, 33,  88,  237, 149, 56,  87,  174, 20,  125, 136, 171, 168, 68,  175, 74,  165,
    71,  134, 139, 48,  27,  166, 77,  146, 158, 231, 83,  111, 229, 122, 60,  211, 133, 230, 220, 105, 92,  41,
    55,  46,  245, 40,  244, 102, 143, 54,  65,  25,  63,  161, 1,   216, 80,  73,  209, 76,  132, 187, 208, 89,
    18,  169, 200, 196, 135, 130, 116, 188, 159, 86,  164, 100, 109, 198, 173, 186, 3,   64,  52,  217, 226, 250,
    124, 123, 5,   202, 38,  147, 118, 126, 255, 82,  85,  212, 207, 206, 59,  227, 47,  16,  58,  17,  182, 189,
    28,  42,  223, 183, 170, 213, 119, 248, 152, 2,   44,  154, 163, 70,  221, 153, 101, 155, 167, 43,  172, 9,
    129, 22,  39,  253, 19,  98,  108, 110, 79,  113, 224, 232, 178, 185, 112, 104, 218, 246, 97,  228, 251, 34,
    242, 193, 238, 210, 144, 12,  191, 179, 162, 241, 81,  51,  145, 235, 249, 14,  239, 107, 49,  192, 214, 31,
    181, 199, 106, 157, 184, 84,  204, 176, 115, 121, 50,  45,  127, 4,   150, 254, 138, 236, 205, 93,  222, 114,
    67,  29,  24,  72,  243, 141, 128, 195, 78,  66,  215, 61,  156, 180};
__device__ __forceinline__ int perm(int i) { return kPerm[i & 255]; }
__device__ __forceinline__ float fade(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }
__device__ __forceinline__ float plerp(float t, float a, float b) { return a + t * (b - a); }
__device__ __forceinline__ float grad(int hash, float x, float y, float z) {
	const int h = hash & 15;
	const float u = h < 8 ? x : y;
	const float v = h < 4 ? y : (h == 12 || h == 14 ? x : z);
	return ((h & 1) == 0 ? u : -u) + ((h & 2) == 0 ? v : -v);
}
__device__ float perlin(float x, float y, float z) {
	const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
	const int X = static_cast<int>(fx) & 255, Y = static_cast<int>(fy) & 255, Z = static_cast<int>(fz) & 255;
	x -= fx;
	y -= fy;
	z -= fz;
	const float u = fade(x), v = fade(y), w = fade(z);
	// The reference indexes a doubled 512-entry table; indices stay below 512.
	const int A = perm(X) + Y, AA = perm(A) + Z, AB = perm(A + 1) + Z;
	const int B = perm(X + 1) + Y, BA = perm(B) + Z, BB = perm(B + 1) + Z;
	return plerp(w,
	             plerp(v, plerp(u, grad(perm(AA), x, y, z), grad(perm(BA), x - 1, y, z)),
	                   plerp(u, grad(perm(AB), x, y - 1, z), grad(perm(BB), x - 1, y - 1, z))),
	             plerp(v, plerp(u, grad(perm(AA + 1), x, y, z - 1), grad(perm(BA + 1), x - 1, y, z - 1)),
	                   plerp(u, grad(perm(AB + 1), x, y - 1, z - 1), grad(perm(BB + 1), x - 1, y - 1, z - 1))));
}
__device__ float fractal_noise(V3 p, int octaves) {
	float sum = 0.0f, amplitude = 1.0f, frequency = 1.0f, norm = 0.0f;
	for (int i = 0; i < octaves; i++) {
		sum += amplitude * perlin(p.x * frequency, p.y * frequency, p.z * frequency);
		norm += amplitude;
		amplitude *= 0.5f;
		frequency *= 2.0f;
	}
	return 0.5f + 0.5f * (sum / norm);
}
__device__ V3 procedural_colour(V3 p) {
	const V3 q = p * 3.0f;
	const float n = fractal_noise(q, 4);
	const float rings = 0.5f + 0.5f * lm_sin((q.x + q.y) * 3.0f + n * 8.0f);
	return mix(mk(60.0f, 30.0f, 12.0f), mk(205.0f, 150.0f, 90.0f), rings);
}

struct Ctx {
	SceneView sv;
	const float4 *ref_shade;
	const RefParams *p;
	int err;
};

struct Hit {
	bool hit;
	int idx;
	float t;
	V3 point;
};

__device__ __forceinline__ Hit intersect(Ctx &c, V3 o, V3 d, int ignore) {
	const RayPre r = make_ray(o.x, o.y, o.z, d.x, d.y, d.z);
	const HitRec h = trace_closest_best<kOrderReference>(c.sv, r, ignore, c.err);
	Hit out;
	out.hit = h.idx >= 0;
	out.idx = h.idx;
	out.t = h.t;
	out.point = o + h.t * d;
	return out;
}
__device__ __forceinline__ bool occluded(Ctx &c, V3 o, V3 d, float maxd, int ignore) {
	const RayPre r = make_ray(o.x, o.y, o.z, d.x, d.y, d.z);
	return trace_any_best(c.sv, r, maxd, ignore, c.err);
}

__device__ __forceinline__ V3 l3(const float *a) { return mk(a[0], a[1], a[2]); }

// The shadow-ray patterns of visibility (src/Renderer.cpp:390-498) one tap at a
// time, for renderers that trace the taps in a separate pass: a light's taps and,
// for tap k, the direction and length of its ray from the shading point, each
// formed with the reference's operations (the same rays visibility() below traces
// in its per-pattern loops).
struct VisTaps {
	int kind; // 0 single ray, 1 rectangle, 2 triangle, 3 volume cone, 4 disk
	int n;
	bool all_visible; // volume light enclosing the point: visibility 1 without rays
	V3 pos, a, b, dir; // rectangle/triangle: u, v axes; disk and volume: tangent, bitangent
	float d, ct0, st0, ct1, st1, radius;
};

// Taps per light for the pattern of light L (the count does not depend on the point).
__device__ __forceinline__ int vis_tap_count(const RefLight &L) { return ref_tap_count(L); }

__device__ __forceinline__ VisTaps vis_taps(const RefLight &L, V3 point) {
	VisTaps T;
	T.all_visible = false;
	T.n = vis_tap_count(L);
	T.pos = l3(L.position);
	if (L.type == kLightDirectional) {
		T.kind = 0;
		T.dir = -normalize(l3(L.direction));
		T.d = 1e6f;
		return T;
	}
	if (L.type == kLightRectangle || L.type == kLightTriangle) {
		T.kind = L.type == kLightRectangle ? 1 : 2;
		T.a = l3(L.u_axis);
		T.b = l3(L.v_axis);
		return T;
	}
	if (L.radius <= 0.0f) {
		T.kind = 0;
		const V3 to = T.pos - point;
		T.d = length(to);
		T.dir = to / T.d;
		return T;
	}
	if (L.type == kLightVolume) {
		T.kind = 3;
		const V3 toc = T.pos - point;
		T.d = length(toc);
		T.dir = toc / T.d;
		const float sin_max = smin(1.0f, L.radius / T.d);
		if (sin_max >= 1.0f) {
			T.all_visible = true;
			return T;
		}
		const float cos_max = sqrtf(smax(0.0f, 1.0f - sin_max * sin_max));
		const V3 up = fabsf(T.dir.y) < 0.99f ? mk(0, 1, 0) : mk(1, 0, 0);
		T.a = normalize(cross(up, T.dir));
		T.b = cross(T.dir, T.a);
		T.ct0 = 1.0f - 0.85f * (1.0f - cos_max);
		T.st0 = sqrtf(smax(0.0f, 1.0f - T.ct0 * T.ct0));
		T.ct1 = 1.0f - 0.4f * (1.0f - cos_max);
		T.st1 = sqrtf(smax(0.0f, 1.0f - T.ct1 * T.ct1));
		return T;
	}
	// Disk light: fixed 9-point pattern (src/Renderer.cpp:483-497).
	T.kind = 4;
	T.radius = L.radius;
	const V3 axis = normalize(point - T.pos);
	const V3 up = fabsf(axis.y) < 0.99f ? mk(0, 1, 0) : mk(1, 0, 0);
	T.a = normalize(cross(up, axis));
	T.b = cross(axis, T.a);
	return T;
}

__device__ __forceinline__ void vis_tap(const VisTaps &T, V3 point, int k, V3 &dir, float &dist) {
	if (T.kind == 0) {
		dir = T.dir;
		dist = T.d;
		return;
	}
	if (T.kind == 3) {
		if (k == 0) {
			dir = T.dir;
		} else {
			// rings of 5 (offset 0) and 6 (offset 0.5) directions
			const float kPi = 3.14159265358979323846f;
			const bool outer = k > 5;
			const int i = outer ? k - 6 : k - 1;
			const int count = outer ? 6 : 5;
			const float off = outer ? 0.5f : 0.0f;
			const float ct = outer ? T.ct1 : T.ct0, st = outer ? T.st1 : T.st0;
			const float phi = 2.0f * kPi * ((static_cast<float>(i) + off) / static_cast<float>(count));
			const V3 sd = T.dir * ct + (T.a * lm_cos(phi) + T.b * lm_sin(phi)) * st;
			dir = normalize(sd);
		}
		dist = T.d;
		return;
	}
	V3 sp;
	if (T.kind == 1) {
		const float gx = static_cast<float>(k % 3 - 1), gy = static_cast<float>(k / 3 - 1);
		sp = T.pos + T.a * gx + T.b * gy;
	} else if (T.kind == 2) {
		const float bx[9] = {0.0f, 1.0f, 0.0f, 0.5f, 0.0f, 0.5f, 0.25f, 0.5f, 1.0f / 3.0f};
		const float by[9] = {0.0f, 0.0f, 1.0f, 0.0f, 0.5f, 0.5f, 0.25f, 0.25f, 1.0f / 3.0f};
		sp = T.pos + T.a * bx[k] + T.b * by[k];
	} else {
		const float sx[9] = {0, 1, -1, 0, 0, 0.7f, -0.7f, 0.7f, -0.7f};
		const float sy[9] = {0, 0, 0, 1, -1, 0.7f, 0.7f, -0.7f, -0.7f};
		sp = T.pos + (T.a * sx[k] + T.b * sy[k]) * T.radius;
	}
	const V3 to = sp - point;
	dist = length(to);
	dir = to / dist;
}

// visibility from the number of unoccluded taps: unocc / 9.0f, unocc / 12 or the
// single ray's 0 / 1, as the reference divides.
__device__ __forceinline__ float vis_fraction(int unocc, int n) {
	return static_cast<float>(unocc) / static_cast<float>(n);
}

// src/Renderer.cpp:390-498
__device__ float visibility(Ctx &c, const RefLight &L, V3 point, int ignore) {
	if (L.type == kLightDirectional) {
		const V3 dir = -normalize(l3(L.direction));
		return occluded(c, point, dir, 1e6f, ignore) ? 0.0f : 1.0f;
	}
	const V3 pos = l3(L.position);
	if (L.type == kLightRectangle) {
		const float gx[9] = {-1, 0, 1, -1, 0, 1, -1, 0, 1};
		const float gy[9] = {-1, -1, -1, 0, 0, 0, 1, 1, 1};
		int unocc = 0;
		for (int k = 0; k < 9; k++) {
			const V3 sp = pos + l3(L.u_axis) * gx[k] + l3(L.v_axis) * gy[k];
			const V3 to = sp - point;
			const float dist = length(to);
			if (!occluded(c, point, to / dist, dist, ignore))
				unocc++;
		}
		return static_cast<float>(unocc) / 9.0f;
	}
	if (L.type == kLightTriangle) {
		const float bx[9] = {0.0f, 1.0f, 0.0f, 0.5f, 0.0f, 0.5f, 0.25f, 0.5f, 1.0f / 3.0f};
		const float by[9] = {0.0f, 0.0f, 1.0f, 0.0f, 0.5f, 0.5f, 0.25f, 0.25f, 1.0f / 3.0f};
		int unocc = 0;
		for (int k = 0; k < 9; k++) {
			const V3 sp = pos + l3(L.u_axis) * bx[k] + l3(L.v_axis) * by[k];
			const V3 to = sp - point;
			const float dist = length(to);
			if (!occluded(c, point, to / dist, dist, ignore))
				unocc++;
		}
		return static_cast<float>(unocc) / 9.0f;
	}
	if (L.radius <= 0.0f) {
		const V3 to = pos - point;
		const float dist = length(to);
		return occluded(c, point, to / dist, dist, ignore) ? 0.0f : 1.0f;
	}
	if (L.type == kLightVolume) {
		const float kPi = 3.14159265358979323846f;
		const V3 toc = pos - point;
		const float d = length(toc);
		const V3 dir = toc / d;
		const float sin_max = smin(1.0f, L.radius / d);
		if (sin_max >= 1.0f)
			return 1.0f;
		const float cos_max = sqrtf(smax(0.0f, 1.0f - sin_max * sin_max));
		const V3 up = fabsf(dir.y) < 0.99f ? mk(0, 1, 0) : mk(1, 0, 0);
		const V3 tangent = normalize(cross(up, dir));
		const V3 bitangent = cross(dir, tangent);
		const float ring_cos[2] = {0.85f, 0.4f};
		const int ring_count[2] = {5, 6};
		const float ring_off[2] = {0.0f, 0.5f};
		int unocc = 0, total = 1;
		if (!occluded(c, point, dir, d, ignore))
			unocc++;
		for (int ring = 0; ring < 2; ring++) {
			const float ct = 1.0f - ring_cos[ring] * (1.0f - cos_max);
			const float st = sqrtf(smax(0.0f, 1.0f - ct * ct));
			const int count = ring_count[ring];
			for (int i = 0; i < count; i++) {
				const float phi =
				    2.0f * kPi * ((static_cast<float>(i) + ring_off[ring]) / static_cast<float>(count));
				V3 sd = dir * ct + (tangent * lm_cos(phi) + bitangent * lm_sin(phi)) * st;
				sd = normalize(sd);
				if (!occluded(c, point, sd, d, ignore))
					unocc++;
				total++;
			}
		}
		return static_cast<float>(unocc) / static_cast<float>(total);
	}
	// Disk light: fixed 9-point pattern (src/Renderer.cpp:483-497).
	const float sx[9] = {0, 1, -1, 0, 0, 0.7f, -0.7f, 0.7f, -0.7f};
	const float sy[9] = {0, 0, 0, 1, -1, 0.7f, 0.7f, -0.7f, -0.7f};
	const V3 axis = normalize(point - pos);
	const V3 up = fabsf(axis.y) < 0.99f ? mk(0, 1, 0) : mk(1, 0, 0);
	const V3 tangent = normalize(cross(up, axis));
	const V3 bitangent = cross(axis, tangent);
	int unocc = 0;
	for (int k = 0; k < 9; k++) {
		const V3 sp = pos + (tangent * sx[k] + bitangent * sy[k]) * L.radius;
		const V3 to = sp - point;
		const float dist = length(to);
		if (!occluded(c, point, to / dist, dist, ignore))
			unocc++;
	}
	return static_cast<float>(unocc) / 9.0f;
}

// Attenuated light direction / falloff shared by directLight and the subsurface branch.
__device__ __forceinline__ void light_dir(const RefLight &L, V3 point, V3 &dir, float &atten) {
	if (L.type == kLightDirectional) {
		dir = -normalize(l3(L.direction));
		atten = L.intensity / 40.0f;
	} else {
		const V3 to = l3(L.position) - point;
		const float dist = length(to);
		dir = to / dist;
		atten = L.intensity / (L.atten_constant + L.atten_linear * dist + L.atten_quadratic * dist * dist);
	}
}

// src/Renderer.cpp:791-814
__device__ V3 direct_light(Ctx &c, V3 point, V3 normal, V3 albedo, int ignore) {
	V3 sum = mk(0, 0, 0);
	for (int li = 0; li < c.p->num_lights; li++) {
		const RefLight &L = c.p->lights[li];
		V3 ld;
		float atten;
		light_dir(L, point, ld, atten);
		float cone = 1.0f;
		if (L.type == kLightSpot)
			cone = (dot(-ld, normalize(l3(L.direction))) > L.cone_cos) ? 1.0f : 0.0f;
		const float vis = visibility(c, L, point, ignore);
		const float incidence = smax(0.0f, dot(normal, ld));
		sum = sum + l3(L.colour) * (vis * cone * atten * incidence);
	}
	return albedo * vmin(sum, mk(1.0f, 1.0f, 1.0f));
}

// src/Renderer.cpp:778-788
// libstdc++ uniform_real_distribution<float>(0, 1) of one 32-bit engine output.
__device__ __forceinline__ float canonical01(uint32_t x) {
	float c = __uint2float_rn(x) / 4294967296.0f;
	if (c >= 1.0f)
		c = 0.99999994f;
	return c * (1.0f - 0.0f) + 0.0f;
}

__device__ V3 cosine_hemisphere_u(V3 n, float u1, float u2) {
	const float r = sqrtf(u1);
	const float theta = 2.0f * 3.14159265f * u2;
	const float x = r * lm_cos(theta), y = r * lm_sin(theta), z = sqrtf(smax(0.0f, 1.0f - u1));
	const V3 up = fabsf(n.z) < 0.99f ? mk(0, 0, 1) : mk(1, 0, 0);
	const V3 t = normalize(cross(up, n));
	const V3 b = cross(n, t);
	return normalize(t * x + b * y + n * z);
}

template <class Rng> __device__ V3 cosine_hemisphere(V3 n, Rng &rng) {
	const float u1 = rng.uniform(0.0f, 1.0f), u2 = rng.uniform(0.0f, 1.0f);
	return cosine_hemisphere_u(n, u1, u2);
}

// src/Renderer.cpp:555-563, gradient sky (the physical sky is off by default).
__device__ __forceinline__ V3 environment(V3 d) {
	const float t = 0.5f * (d.y + 1.0f);
	return mix(mk(200.0f, 210.0f, 235.0f), mk(70.0f, 120.0f, 205.0f), t);
}

// src/Renderer.cpp:642-660 (flat colour and procedural branches).
__device__ __forceinline__ V3 base_colour(int material, V3 rgb, V3 point) {
	if (material == kRefProcedural)
		return procedural_colour(point);
	return rgb;
}


// x86-64 float -> int conversion (cvttss2si): out-of-range and NaN give INT_MIN.
__device__ __forceinline__ int cvt_trunc(float v) {
	return (v >= -2147483648.0f && v < 2147483648.0f) ? static_cast<int>(v) : static_cast<int>(0x80000000u);
}


} // namespace
} // namespace rnb
