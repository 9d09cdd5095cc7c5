// Reference-mode path tracer: the drop-in behind rn_render(RN_PATHTRACED).
//
// It evaluates the reference estimator (src/Renderer.cpp:775-907, 1103-1170)
// on the GPU, one thread per pixel:
//   * per-pixel std::mt19937 stream seeded (y*W + x)*9781 + 1 and drawn through
//     libstdc++'s uniform_real_distribution<float> (one 32-bit draw per value,
//     float(x) / 2^32), in the reference's draw order, so every pixel consumes the
//     same random numbers as the CPU renderer;
//   * the recursive pathTrace is unrolled into a short frame stack and folded back
//     from the deepest level, so radiance is combined in the reference's order;
//   * this file is compiled with -fmad=false: single-precision expressions are
//     evaluated as separately rounded IEEE operations in source order, matching the
//     reference's non-FMA x86-64 build; sin/cos/pow/exp are evaluated in double and
//     rounded once to float (the correctly rounded value the host libm returns in
//     all but rare cases);
//   * closest hit / occlusion use the reference-order traversal (traverse.cuh).
// Per pixel the output is then the reference's 8-bit value except where a libm
// last-bit difference moves a path or a truncation boundary.
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
__device__ V3 cosine_hemisphere(V3 n, MT &rng) {
	const float u1 = rng.uniform(0.0f, 1.0f), u2 = rng.uniform(0.0f, 1.0f);
	const float r = sqrtf(u1);
	const float theta = 2.0f * 3.14159265f * u2;
	const float x = r * lm_cos(theta), y = r * lm_sin(theta), z = sqrtf(smax(0.0f, 1.0f - u1));
	const V3 up = fabsf(n.z) < 0.99f ? mk(0, 0, 1) : mk(1, 0, 0);
	const V3 t = normalize(cross(up, n));
	const V3 b = cross(n, t);
	return normalize(t * x + b * y + n * z);
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

constexpr int kMaxLevels = kMaxRefDepth + 1; // recursion levels max_depth..0

// One pathTrace(origin, dir, depth = max_depth) evaluation (src/Renderer.cpp:820-907),
// unrolled: each level records R_k = add + mul * R_{k+1} (kind 2), mul * R_{k+1}
// (kind 1) or R_{k+1} (kind 0), then the levels are folded deepest first.
__device__ V3 path_trace(Ctx &c, V3 origin, V3 direction, MT &rng) {
	V3 add[kMaxLevels], mul[kMaxLevels];
	int kind[kMaxLevels];
	int levels = 0;
	V3 result = mk(0, 0, 0);
	int depth = c.p->max_depth;
	for (;;) {
		const Hit hit = intersect(c, origin, direction, -1);
		if (!hit.hit) {
			result = environment(direction) / 255.0f;
			break;
		}
		const float4 s0 = __ldg(c.ref_shade + 2 * static_cast<size_t>(hit.idx));
		const float4 s1 = __ldg(c.ref_shade + 2 * static_cast<size_t>(hit.idx) + 1);
		const V3 tnormal = mk(s0.x, s0.y, s0.z);
		const int material = __float_as_int(s0.w);
		const V3 rgb = mk(s1.x, s1.y, s1.z);
		const float roughness = s1.w;
		const V3 point = hit.point;
		const int ignore = hit.idx;
		if (material == kRefEmissive) {
			result = rgb / 255.0f * 4.0f;
			break;
		}
		if (material == kRefMirror && depth > 0) {
			const V3 n = face_viewer(tnormal, direction);
			const V3 refl = reflect(direction, n);
			kind[levels++] = 0;
			origin = point + 1e-4f * refl;
			direction = refl;
			depth--;
			continue;
		}
		if ((material == kRefGlass || material == kRefDispersive) && depth > 0) {
			const float ior = 1.5f;
			V3 n = tnormal;
			float cosi = dot(direction, n);
			float etai = 1.0f, etat = ior;
			if (cosi < 0.0f) {
				cosi = -cosi;
			} else {
				const float tmp = etai;
				etai = etat;
				etat = tmp;
				n = -n;
			}
			float r0 = (etai - etat) / (etai + etat);
			r0 *= r0;
			const float fresnel = r0 + (1.0f - r0) * lm_pow(1.0f - cosi, 5.0f);
			const V3 refr = refract(direction, n, etai / etat);
			bool do_reflect = length(refr) < 1e-6f;
			if (!do_reflect)
				do_reflect = rng.uniform(0.0f, 1.0f) < fresnel;
			const V3 dir = do_reflect ? reflect(direction, n) : refr;
			kind[levels++] = 0;
			origin = point + 1e-4f * dir;
			direction = dir;
			depth--;
			continue;
		}
		if (material == kRefMetal && depth > 0) {
			const V3 n = face_viewer(tnormal, direction);
			const V3 refl = reflect(direction, n);
			const V3 diff = cosine_hemisphere(n, rng);
			const float r2 = roughness * roughness;
			V3 dir = normalize(mix(refl, diff, r2));
			if (dot(dir, n) <= 0.0f)
				dir = refl;
			const V3 albedo = base_colour(material, rgb, point) / 255.0f;
			mul[levels] = albedo;
			kind[levels++] = 1;
			origin = point + 1e-4f * dir;
			direction = dir;
			depth--;
			continue;
		}
		if (material == kRefSubsurface) {
			const V3 n = face_viewer(tnormal, direction);
			const V3 albedo = base_colour(material, rgb, point) / 255.0f;
			V3 shade = mk(0, 0, 0);
			const float wrap = 0.5f;
			for (int li = 0; li < c.p->num_lights; li++) {
				const RefLight &L = c.p->lights[li];
				const V3 to = l3(L.position) - point;
				const float dist = length(to);
				const V3 ld = to / dist;
				const float atten =
				    L.intensity / (L.atten_constant + L.atten_linear * dist + L.atten_quadratic * dist * dist);
				const float wrap_diff = smax(0.0f, (dot(n, ld) + wrap) / (1.0f + wrap));
				shade = shade + albedo * l3(L.colour) * (visibility(c, L, point, ignore) * atten * wrap_diff);
				const Hit ex = intersect(c, point - n * 1e-3f, ld, ignore);
				const float thickness = ex.hit ? ex.t : 0.0f;
				shade = shade + albedo * l3(L.colour) * (atten * lm_exp(-3.0f * thickness) * 0.6f);
			}
			const V3 direct = vmin(shade, mk(1.5f, 1.5f, 1.5f));
			if (depth <= 0) {
				result = direct;
				break;
			}
			const V3 sb = cosine_hemisphere(n, rng);
			add[levels] = direct;
			mul[levels] = albedo;
			kind[levels++] = 2;
			origin = point + 1e-4f * sb;
			direction = sb;
			depth--;
			continue;
		}
		// Diffuse (and every branch above once depth reaches 0).
		const V3 n = face_viewer(tnormal, direction);
		const V3 albedo = base_colour(material, rgb, point) / 255.0f;
		const V3 direct = direct_light(c, point, n, albedo, ignore);
		if (depth <= 0) {
			result = direct;
			break;
		}
		const V3 bounce = cosine_hemisphere(n, rng);
		add[levels] = direct;
		mul[levels] = albedo;
		kind[levels++] = 2;
		origin = point + 1e-4f * bounce;
		direction = bounce;
		depth--;
	}
	for (int k = levels - 1; k >= 0; k--) {
		if (kind[k] == 2)
			result = add[k] + mul[k] * result;
		else if (kind[k] == 1)
			result = mul[k] * result;
	}
	return result;
}

// src/Renderer.cpp:1103-1117
__device__ void sample_aperture(int blades, float u1, float u2, float &lx, float &ly) {
	if (blades < 3) {
		const float ang = 2.0f * 3.14159265f * u1, rad = sqrtf(u2);
		lx = lm_cos(ang) * rad;
		ly = lm_sin(ang) * rad;
		return;
	}
	const int wedge = min(blades - 1, static_cast<int>(u1 * blades));
	const float a0 = 2.0f * 3.14159265f * wedge / blades, a1 = 2.0f * 3.14159265f * (wedge + 1) / blades;
	const float v0x = lm_cos(a0), v0y = lm_sin(a0), v1x = lm_cos(a1), v1y = lm_sin(a1);
	float s = u1 * blades - wedge, t = u2;
	if (s + t > 1.0f) {
		s = 1.0f - s;
		t = 1.0f - t;
	}
	lx = v0x * s + v1x * t;
	ly = v0y * s + v1y * t;
}

// x86-64 float -> int conversion (cvttss2si): out-of-range and NaN give INT_MIN.
__device__ __forceinline__ int cvt_trunc(float v) {
	return (v >= -2147483648.0f && v < 2147483648.0f) ? static_cast<int>(v) : static_cast<int>(0x80000000u);
}

__global__ void __launch_bounds__(128) k_render_reference(SceneView sv, const float4 *__restrict__ ref_shade,
                                                          const RefParams *__restrict__ params,
                                                          uint32_t *__restrict__ argb, float *__restrict__ mean_rgb,
                                                          int *status) {
	const RefParams &p = *params;
	const long pix = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (pix >= static_cast<long>(p.width) * p.height)
		return;
	const int x = static_cast<int>(pix % p.width), y = static_cast<int>(pix / p.width);
	Ctx c{sv, ref_shade, &p, 0};
	MT rng;
	rng.seed(static_cast<uint32_t>((static_cast<uint32_t>(y) * static_cast<uint32_t>(p.width) +
	                                static_cast<uint32_t>(x)) *
	                                   9781u +
	                               1u));
	const V3 right = mk(p.orient[0], p.orient[1], p.orient[2]);
	const V3 upv = mk(p.orient[3], p.orient[4], p.orient[5]);
	const V3 fwd = mk(p.orient[6], p.orient[7], p.orient[8]);
	const V3 pos = l3(p.position);
	const V3 motion = l3(p.camera_motion);
	const float f = p.f;
	V3 sum = mk(0, 0, 0);
	for (int s = 0; s < p.samples; s++) {
		const float jx = rng.uniform(-0.5f, 0.5f);
		const float jy = rng.uniform(-0.5f, 0.5f);
		const float sx = static_cast<float>(x) + 0.5f + jx - static_cast<float>(p.width) / 2.0f;
		const float sy = -(static_cast<float>(y) + 0.5f + jy - static_cast<float>(p.height) / 2.0f);
		V3 ro, dir;
		if (p.orthographic) {
			const V3 v = mk(sx / f * p.ortho_scale, sy / f * p.ortho_scale, 0.0f);
			ro = pos + (right * v.x + upv * v.y + fwd * v.z);
			dir = normalize(right * 0.0f + upv * 0.0f + fwd * -1.0f);
		} else {
			const V3 v = mk(sx / f, sy / f, -1.0f);
			ro = pos;
			dir = normalize(right * v.x + upv * v.y + fwd * v.z);
		}
		const V3 cam = ro + motion * rng.uniform(0.0f, 1.0f);
		V3 origin = cam;
		if (p.aperture > 0.0f && !p.orthographic) {
			const V3 focal = cam + dir * p.focus_distance;
			// sampleAperture(blades, U(rng), U(rng)): GCC evaluates these two call
			// arguments right to left, so the second argument is drawn first.
			float ua, ub;
			if (p.aperture_args_right_to_left) {
				ub = rng.uniform(0.0f, 1.0f);
				ua = rng.uniform(0.0f, 1.0f);
			} else {
				ua = rng.uniform(0.0f, 1.0f);
				ub = rng.uniform(0.0f, 1.0f);
			}
			float lx, ly;
			sample_aperture(p.aperture_blades, ua, ub, lx, ly);
			lx = lx * p.aperture;
			ly = ly * p.aperture;
			origin = cam + (right * lx + upv * ly);
			dir = normalize(focal - origin);
		}
		sum = sum + path_trace(c, origin, dir, rng);
	}
	const V3 colour = sum / static_cast<float>(p.samples) * 255.0f;
	const int r = min(255, cvt_trunc(colour.x));
	const int g = min(255, cvt_trunc(colour.y));
	const int b = min(255, cvt_trunc(colour.z));
	argb[pix] = (255u << 24) | ((static_cast<uint32_t>(r) & 0xFFu) << 16) | ((static_cast<uint32_t>(g) & 0xFFu) << 8) |
	            (static_cast<uint32_t>(b) & 0xFFu);
	if (mean_rgb) {
		const V3 m = sum / static_cast<float>(p.samples);
		mean_rgb[3 * pix] = m.x;
		mean_rgb[3 * pix + 1] = m.y;
		mean_rgb[3 * pix + 2] = m.z;
	}
	if (c.err)
		atomicOr(status, 1);
}

// ---- Whitted ray tracing (renderRaytraced, src/Renderer.cpp:500-773 and 909-948) ----

struct WHit {
	bool hit;
	int idx;
	float t, u, v;
	V3 point;
};
__device__ __forceinline__ WHit intersect_uv(Ctx &c, V3 o, V3 d) {
	const RayPre r = make_ray(o.x, o.y, o.z, d.x, d.y, d.z);
	const HitRec h = trace_closest_best<kOrderReference>(c.sv, r, -1, c.err);
	WHit out;
	out.hit = h.idx >= 0;
	out.idx = h.idx;
	out.t = h.t;
	out.u = h.u;
	out.v = h.v;
	out.point = o + h.t * d;
	return out;
}

// shadeSurface (src/Renderer.cpp:503-535): per light, proximity/incidence diffuse and
// a power-64 specular lobe, both times soft-shadow visibility, on an ambient floor.
__device__ V3 shade_surface(Ctx &c, V3 point, V3 normal, V3 view_dir, int ignore, V3 base) {
	const float ambient = 0.2f;
	V3 diffuse = mk(0.0f, 0.0f, 0.0f);
	float spec = 0.0f;
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
		const float brightness = vis * cone * atten * incidence;
		diffuse = diffuse + l3(L.colour) * brightness;
		if (brightness > 0.0f) {
			const V3 rd = (2.0f * dot(normal, ld)) * normal - ld;
			spec += vis * cone * lm_pow(smax(0.0f, dot(rd, view_dir)), 64.0f);
		}
	}
	const V3 lit = vmin(mk(1.0f, 1.0f, 1.0f), diffuse + mk(ambient, ambient, ambient));
	return base * lit + mk(255.0f, 255.0f, 255.0f) * smin(1.0f, spec);
}

// bumpNormal (src/Renderer.cpp:574-581): the normal tilted by a Perlin gradient.
__device__ V3 bump_normal(V3 normal, V3 p) {
	const V3 q = p * 6.0f;
	const float e = 0.15f;
	const V3 g = mk(perlin(q.x + e, q.y, q.z) - perlin(q.x - e, q.y, q.z),
	                perlin(q.x, q.y + e, q.z) - perlin(q.x, q.y - e, q.z),
	                perlin(q.x, q.y, q.z + e) - perlin(q.x, q.y, q.z - e));
	return normalize(normal + 2.0f * g);
}

// shadeDiffuse (src/Renderer.cpp:663-700), untextured: flat, Gouraud or Phong.
__device__ V3 shade_diffuse(Ctx &c, const float4 *__restrict__ geom, const WHit &hit, V3 dir) {
	const float4 s0 = c.ref_shade[2 * hit.idx], s1 = c.ref_shade[2 * hit.idx + 1];
	const int mat = __float_as_int(s0.w);
	const V3 point = hit.point;
	const V3 view = -dir;
	const float w0 = 1.0f - hit.u - hit.v, w1 = hit.u, w2 = hit.v;
	const V3 base = base_colour(mat, mk(s1.x, s1.y, s1.z), point);
	const float4 *g = geom + 6 * static_cast<size_t>(hit.idx);
	if (c.p->shading == 1) { // Gouraud: shade the corners, interpolate the colours
		V3 col[3];
		for (int k = 0; k < 3; k++) {
			const float4 vk = g[k], nk = g[3 + k];
			col[k] = shade_surface(c, mk(vk.x, vk.y, vk.z), face_viewer(mk(nk.x, nk.y, nk.z), dir), view, hit.idx,
			                       base);
		}
		return w0 * col[0] + w1 * col[1] + w2 * col[2];
	}
	V3 normal;
	if (c.p->shading == 2) {
		const float4 n0 = g[3], n1 = g[4], n2 = g[5];
		normal = normalize(w0 * mk(n0.x, n0.y, n0.z) + w1 * mk(n1.x, n1.y, n1.z) + w2 * mk(n2.x, n2.y, n2.z));
	} else {
		normal = mk(s0.x, s0.y, s0.z);
	}
	normal = face_viewer(normal, dir);
	if (mat == kRefBump)
		normal = bump_normal(normal, point);
	return shade_surface(c, point, normal, view, hit.idx, base);
}

// traceRay's recursion (src/Renderer.cpp:704-773) on an explicit stack. A frame is a
// traceRay call whose value combines the values of its child rays: one reflection
// for mirrors and metal, and per glassTrace (one for glass, three indices of
// refraction for dispersive glass) a reflection and, unless totally reflected, a
// refraction. Each value is formed from its children exactly as the reference
// forms it, so the result is the recursion's, bit for bit.
constexpr int kWMirror = 0, kWMetal = 1, kWGlass = 2;
struct WFrame {
	V3 co[6], cd[6], res[6];
	V3 tint;
	float fres[3];
	int n, next, kind, ng, tir, depth;
};

// glassTrace's rays and Fresnel weight (src/Renderer.cpp:711-731) for child pair g.
__device__ void glass_setup(V3 point, V3 direction, V3 tri_n, float ior, WFrame &f, int g) {
	V3 n = tri_n;
	float cosi = dot(direction, n);
	float etai = 1.0f, etat = ior;
	if (cosi < 0.0f) {
		cosi = -cosi;
	} else {
		const float tmp = etai;
		etai = etat;
		etat = tmp;
		n = -n;
	}
	const V3 refl = reflect(direction, n);
	f.co[2 * g] = point + 1e-4f * refl;
	f.cd[2 * g] = refl;
	const V3 refr = refract(direction, n, etai / etat);
	f.fres[g] = 0.0f;
	if (length(refr) < 1e-6f) {
		f.tir |= 1 << g;
		return;
	}
	float r0 = (etai - etat) / (etai + etat);
	r0 *= r0;
	f.fres[g] = r0 + (1.0f - r0) * lm_pow(1.0f - cosi, 5.0f);
	f.co[2 * g + 1] = point + 1e-4f * refr;
	f.cd[2 * g + 1] = refr;
}

// One traceRay(o, d, depth): its value (true), or the frame of its child rays (false).
__device__ bool whitted_expand(Ctx &c, const float4 *__restrict__ geom, V3 o, V3 d, int depth, V3 &value,
                               WFrame &f) {
	const WHit hit = intersect_uv(c, o, d);
	if (!hit.hit) {
		value = environment(d);
		return true;
	}
	const float4 s0 = c.ref_shade[2 * hit.idx], s1 = c.ref_shade[2 * hit.idx + 1];
	const int mat = __float_as_int(s0.w);
	const V3 tri_n = mk(s0.x, s0.y, s0.z), rgb = mk(s1.x, s1.y, s1.z);
	if (mat == kRefEmissive) {
		value = rgb * 1.3f;
		return true;
	}
	if (depth > 0 && (mat == kRefMirror || mat == kRefMetal)) {
		const V3 n = face_viewer(tri_n, d);
		const V3 r = reflect(d, n);
		f.co[0] = hit.point + 1e-4f * r;
		f.cd[0] = r;
		f.n = 1;
		f.next = 0;
		f.kind = mat == kRefMirror ? kWMirror : kWMetal;
		f.tint = rgb / 255.0f;
		f.ng = 0;
		f.tir = 0;
		f.depth = depth;
		return false;
	}
	if (depth > 0 && (mat == kRefGlass || mat == kRefDispersive)) {
		f.kind = kWGlass;
		f.ng = mat == kRefGlass ? 1 : 3;
		f.n = 2 * f.ng;
		f.next = 0;
		f.tir = 0;
		f.depth = depth;
		if (f.ng == 1) {
			glass_setup(hit.point, d, tri_n, 1.5f, f, 0);
		} else {
			glass_setup(hit.point, d, tri_n, 1.50f, f, 0);
			glass_setup(hit.point, d, tri_n, 1.53f, f, 1);
			glass_setup(hit.point, d, tri_n, 1.56f, f, 2);
		}
		return false;
	}
	value = shade_diffuse(c, geom, hit, d);
	return true;
}

__device__ V3 whitted_combine(const WFrame &f) {
	if (f.kind == kWMirror)
		return f.res[0];
	if (f.kind == kWMetal)
		return f.tint * f.res[0];
	V3 g[3];
	for (int k = 0; k < f.ng; k++)
		g[k] = ((f.tir >> k) & 1) ? f.res[2 * k] : f.fres[k] * f.res[2 * k] + (1.0f - f.fres[k]) * f.res[2 * k + 1];
	if (f.ng == 1)
		return g[0];
	return mk(g[0].x, g[1].y, g[2].z);
}

__device__ V3 trace_whitted(Ctx &c, const float4 *__restrict__ geom, V3 o, V3 d, int max_depth) {
	// Frames have depth >= 1 and a child's depth is one less, so at most max_depth
	// frames are open at once.
	WFrame st[kMaxWhittedDepth + 1];
	V3 v;
	if (whitted_expand(c, geom, o, d, max_depth, v, st[0]))
		return v;
	int sp = 1;
	for (;;) {
		WFrame &f = st[sp - 1];
		while (f.next < f.n && f.kind == kWGlass && (f.next & 1) && ((f.tir >> (f.next >> 1)) & 1))
			f.next++; // no refraction ray after total internal reflection
		if (f.next < f.n) {
			const int i = f.next;
			if (whitted_expand(c, geom, f.co[i], f.cd[i], f.depth - 1, v, st[sp])) {
				f.res[i] = v;
				f.next++;
			} else {
				sp++;
			}
			continue;
		}
		v = whitted_combine(f);
		if (--sp == 0)
			return v;
		WFrame &parent = st[sp - 1];
		parent.res[parent.next] = v;
		parent.next++;
	}
}

__global__ void __launch_bounds__(128) k_render_raytraced(SceneView sv, const float4 *__restrict__ ref_shade,
                                                          const float4 *__restrict__ geom,
                                                          const RefParams *__restrict__ params,
                                                          uint32_t *__restrict__ argb, int *status) {
	const RefParams &p = *params;
	const long pix = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (pix >= static_cast<long>(p.width) * p.height)
		return;
	const int x = static_cast<int>(pix % p.width), y = static_cast<int>(pix / p.width);
	Ctx c{sv, ref_shade, &p, 0};
	const V3 right = mk(p.orient[0], p.orient[1], p.orient[2]);
	const V3 upv = mk(p.orient[3], p.orient[4], p.orient[5]);
	const V3 fwd = mk(p.orient[6], p.orient[7], p.orient[8]);
	const V3 pos = l3(p.position);
	const float f = p.f;
	// Camera::primaryRay(x - W/2, -(y - H/2), f) (src/Camera.cpp:69-79)
	const float sx = static_cast<float>(x) - static_cast<float>(p.width) / 2.0f;
	const float sy = -(static_cast<float>(y) - static_cast<float>(p.height) / 2.0f);
	V3 ro, dir;
	if (p.orthographic) {
		const V3 v = mk(sx / f * p.ortho_scale, sy / f * p.ortho_scale, 0.0f);
		ro = pos + (right * v.x + upv * v.y + fwd * v.z);
		dir = normalize(right * 0.0f + upv * 0.0f + fwd * -1.0f);
	} else {
		const V3 v = mk(sx / f, sy / f, -1.0f);
		ro = pos;
		dir = normalize(right * v.x + upv * v.y + fwd * v.z);
	}
	V3 colour = trace_whitted(c, geom, ro, dir, p.max_depth);
	if (p.fog_density > 0.0f) {
		const WHit h = intersect_uv(c, ro, dir);
		const float dist = h.hit ? h.t : 30.0f;
		colour = mix(colour, l3(p.fog_colour), 1.0f - lm_exp(-p.fog_density * dist));
	}
	const int r = min(255, cvt_trunc(colour.x));
	const int g = min(255, cvt_trunc(colour.y));
	const int b = min(255, cvt_trunc(colour.z));
	argb[pix] = (255u << 24) | ((static_cast<uint32_t>(r) & 0xFFu) << 16) | ((static_cast<uint32_t>(g) & 0xFFu) << 8) |
	            (static_cast<uint32_t>(b) & 0xFFu);
	if (c.err)
		atomicOr(status, 1);
}

} // namespace

cudaError_t launch_render_raytraced(const SceneView &sv, const float4 *ref_shade, const float4 *ref_geom,
                                    const RefParams *d_params, int width, int height, uint32_t *argb, int *status,
                                    cudaStream_t st) {
	const long n = static_cast<long>(width) * height;
	if (n <= 0)
		return cudaSuccess;
	const int bs = 128;
	k_render_raytraced<<<ceil_div(n, bs), bs, 0, st>>>(sv, ref_shade, ref_geom, d_params, argb, status);
	return cudaGetLastError();
}

cudaError_t launch_render_reference(const SceneView &sv, const float4 *ref_shade, const RefParams *d_params, int width,
                                    int height, uint32_t *argb, float *mean_rgb, int *status, cudaStream_t st) {
	const long n = static_cast<long>(width) * height;
	if (n <= 0)
		return cudaSuccess;
	const int bs = 128;
	k_render_reference<<<ceil_div(n, bs), bs, 0, st>>>(sv, ref_shade, d_params, argb, mean_rgb, status);
	return cudaGetLastError();
}

} // namespace rnb
