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
#include <algorithm>
#include <cstdint>

#include "refshade.cuh"
#include "trace_range.hpp"

namespace rnb {

namespace {

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

struct CamBasis {
	V3 right, upv, fwd, pos, motion;
};
__device__ __forceinline__ CamBasis cam_basis(const RefParams &p) {
	return {mk(p.orient[0], p.orient[1], p.orient[2]), mk(p.orient[3], p.orient[4], p.orient[5]),
	        mk(p.orient[6], p.orient[7], p.orient[8]), l3(p.position), l3(p.camera_motion)};
}

// One camera sample of renderPathTraced's pixel loop (src/Renderer.cpp:1139-1166):
// jitter, orthographic or perspective ray, motion blur, depth of field.
template <class Rng>
__device__ __forceinline__ void camera_sample(const RefParams &p, const CamBasis &b, int x, int y, Rng &rng, V3 &origin,
                                              V3 &dir) {
	const float jx = rng.uniform(-0.5f, 0.5f);
	const float jy = rng.uniform(-0.5f, 0.5f);
	const float sx = static_cast<float>(x) + 0.5f + jx - static_cast<float>(p.width) / 2.0f;
	const float sy = -(static_cast<float>(y) + 0.5f + jy - static_cast<float>(p.height) / 2.0f);
	V3 ro;
	if (p.orthographic) {
		const V3 v = mk(sx / p.f * p.ortho_scale, sy / p.f * p.ortho_scale, 0.0f);
		ro = b.pos + (b.right * v.x + b.upv * v.y + b.fwd * v.z);
		dir = normalize(b.right * 0.0f + b.upv * 0.0f + b.fwd * -1.0f);
	} else {
		const V3 v = mk(sx / p.f, sy / p.f, -1.0f);
		ro = b.pos;
		dir = normalize(b.right * v.x + b.upv * v.y + b.fwd * v.z);
	}
	const V3 cam = ro + b.motion * rng.uniform(0.0f, 1.0f);
	origin = cam;
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
		origin = cam + (b.right * lx + b.upv * ly);
		dir = normalize(focal - origin);
	}
}

__device__ __forceinline__ void store_pixel(long pix, V3 sum, int samples, uint32_t *argb, float *mean_rgb) {
	const V3 colour = sum / static_cast<float>(samples) * 255.0f;
	const int r = min(255, cvt_trunc(colour.x));
	const int g = min(255, cvt_trunc(colour.y));
	const int b = min(255, cvt_trunc(colour.z));
	argb[pix] = (255u << 24) | ((static_cast<uint32_t>(r) & 0xFFu) << 16) | ((static_cast<uint32_t>(g) & 0xFFu) << 8) |
	            (static_cast<uint32_t>(b) & 0xFFu);
	if (mean_rgb) {
		const V3 m = sum / static_cast<float>(samples);
		mean_rgb[3 * pix] = m.x;
		mean_rgb[3 * pix + 1] = m.y;
		mean_rgb[3 * pix + 2] = m.z;
	}
}

__device__ __forceinline__ uint32_t pixel_seed(int x, int y, int width) {
	return static_cast<uint32_t>(
	    (static_cast<uint32_t>(y) * static_cast<uint32_t>(width) + static_cast<uint32_t>(x)) * 9781u + 1u);
}

// ---- the drop-in path tracer in three passes ----
// Visibility draws no random numbers, so a path's vertices do not depend on it:
//  1. k_ref_paths: one thread per pixel walks every sample's path on the pixel's
//     mt19937 stream (closest hits, material choices, bounces) and records each
//     level; levels that need direct light join a compact shading list;
//  2. k_ref_shadow: one thread per (shading entry, light, tap) traces that tap's
//     shadow ray -- the taps of one point sit in adjacent lanes, so a warp's rays
//     leave a few nearby points toward the same light;
//  3. k_ref_fold: one thread per pixel forms directLight (and the subsurface term)
//     from the recorded occlusions with the reference's operations and folds each
//     path from its deepest level, in the reference's order.
// Each level is three float4: (point, kind), (normal, ignore), (albedo or value,
// shading entry).
enum LevelKind : int { kLvPass = 0, kLvMul = 1, kLvDiffuse = 2, kLvSub = 3, kLvDiffuseEnd = 4, kLvSubEnd = 5, kLvValue = 6 };

constexpr int kShadeKeyBits = 15; // 5 bits per axis of the scene box

struct DeferView {
	float4 *rec;
	int *list;
	unsigned *list_count;
	uint8_t *occl;
	unsigned *pix_next; // next pixel of the chunk for the path pass to take
	uint16_t *key;    // per shading entry: Morton cell of its point
	int *sorted;      // shading entries ordered by cell
	unsigned *bins;   // 2^kShadeKeyBits counters, then offsets
	int levels;
	int taps;
	long pix0;
	long npix;
	long cap; // shading entries the chunk's buffers hold
};

__device__ __forceinline__ int shading_append(unsigned *count) {
	const unsigned mask = __activemask();
	const int lane = static_cast<int>(threadIdx.x & 31);
	const int leader = __ffs(mask) - 1;
	unsigned base = 0;
	if (lane == leader)
		base = atomicAdd(count, static_cast<unsigned>(__popc(mask)));
	base = __shfl_sync(mask, base, leader);
	return static_cast<int>(base) + __popc(mask & ((1u << lane) - 1u));
}

__device__ __forceinline__ uint32_t spread5(uint32_t v) {
	v &= 31u;
	v = (v | (v << 8)) & 0x100Fu;
	v = (v | (v << 4)) & 0x10C3u;
	v = (v | (v << 2)) & 0x1249u;
	return v;
}
// 15-bit Morton cell of a point in the scene's root box (5 bits per axis).
__device__ __forceinline__ uint16_t shade_key(const SceneView &sv, V3 p) {
	const float q[3] = {p.x, p.y, p.z};
	uint32_t c[3];
	for (int a = 0; a < 3; a++) {
		const float ext = sv.root_hi[a] - sv.root_lo[a];
		const float f = ext > 0.0f ? (q[a] - sv.root_lo[a]) / ext : 0.0f;
		c[a] = static_cast<uint32_t>(fminf(fmaxf(f * 32.0f, 0.0f), 31.0f));
	}
	return static_cast<uint16_t>(spread5(c[0]) | (spread5(c[1]) << 1) | (spread5(c[2]) << 2));
}

__device__ __forceinline__ void put_level(float4 *r, int kind, V3 a, V3 n, int ignore, V3 b, int entry) {
	r[0] = make_float4(a.x, a.y, a.z, __int_as_float(kind));
	r[1] = make_float4(n.x, n.y, n.z, __int_as_float(ignore));
	r[2] = make_float4(b.x, b.y, b.z, __int_as_float(entry));
}

// pathTrace (src/Renderer.cpp:820-907) without the direct-light terms: the same
// intersections, branches and random draws, recorded level by level.
template <class Rng>
__device__ void record_path(Ctx &c, V3 origin, V3 direction, Rng &rng, const DeferView &dv, size_t rec_index) {
	int depth = c.p->max_depth;
	for (int level = 0; level < dv.levels; level++) {
		float4 *r = dv.rec + 3 * (rec_index + level);
		const V3 zero = mk(0.0f, 0.0f, 0.0f);
		const Hit hit = intersect(c, origin, direction, -1);
		if (!hit.hit) {
			put_level(r, kLvValue, zero, zero, -1, environment(direction) / 255.0f, -1);
			return;
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
			put_level(r, kLvValue, zero, zero, -1, rgb / 255.0f * 4.0f, -1);
			return;
		}
		if (material == kRefMirror && depth > 0) {
			const V3 n = face_viewer(tnormal, direction);
			const V3 refl = reflect(direction, n);
			put_level(r, kLvPass, zero, zero, -1, zero, -1);
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
			put_level(r, kLvPass, zero, zero, -1, zero, -1);
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
			put_level(r, kLvMul, zero, zero, -1, base_colour(material, rgb, point) / 255.0f, -1);
			origin = point + 1e-4f * dir;
			direction = dir;
			depth--;
			continue;
		}
		const bool sub = material == kRefSubsurface;
		const V3 n = face_viewer(tnormal, direction);
		const V3 albedo = base_colour(material, rgb, point) / 255.0f;
		const int entry = shading_append(dv.list_count);
		if (kBoundsCheck && entry >= dv.cap) {
			c.err = 1;
			return;
		}
		dv.list[entry] = static_cast<int>(rec_index + level);
		dv.key[entry] = shade_key(c.sv, point);
		if (depth <= 0) {
			put_level(r, sub ? kLvSubEnd : kLvDiffuseEnd, point, n, ignore, albedo, entry);
			return;
		}
		const V3 bounce = cosine_hemisphere(n, rng);
		put_level(r, sub ? kLvSub : kLvDiffuse, point, n, ignore, albedo, entry);
		origin = point + 1e-4f * bounce;
		direction = bounce;
		depth--;
	}
}

// Persistent: a lane that has finished its pixel takes the next one, so lanes
// whose paths end early do not idle until the warp's longest pixel is done.
__global__ void __launch_bounds__(128) k_ref_paths(SceneView sv, const float4 *__restrict__ ref_shade,
                                                   const RefParams *__restrict__ params, DeferView dv, int *status) {
	const RefParams &p = *params;
	Ctx c{sv, ref_shade, &p, 0};
	const CamBasis b = cam_basis(p);
	for (;;) {
		const long li = atomicAdd(dv.pix_next, 1u);
		if (li >= dv.npix)
			break;
		const long pix = dv.pix0 + li;
		const int x = static_cast<int>(pix % p.width), y = static_cast<int>(pix / p.width);
		MtFresh rng;
		rng.seed(pixel_seed(x, y, p.width));
		for (int s = 0; s < p.samples; s++) {
			V3 origin, dir;
			camera_sample(p, b, x, y, rng, origin, dir);
			record_path(c, origin, dir, rng, dv, (static_cast<size_t>(li) * p.samples + s) * dv.levels);
		}
	}
	if (c.err)
		atomicOr(status, 1);
}

// Counting sort of the shading entries by cell, so that a warp's shadow rays
// start from nearby points.
__global__ void k_shade_count(DeferView dv) {
	const long n = *dv.list_count;
	for (long e = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
	     e += static_cast<long>(gridDim.x) * blockDim.x)
		atomicAdd(dv.bins + dv.key[e], 1u);
}
__global__ void __launch_bounds__(1024) k_shade_scan(DeferView dv) {
	constexpr int kBins = 1 << kShadeKeyBits, kPer = kBins / 1024;
	__shared__ unsigned part[1024];
	const int t = threadIdx.x;
	unsigned sum = 0;
	for (int j = 0; j < kPer; j++)
		sum += dv.bins[t * kPer + j];
	part[t] = sum;
	__syncthreads();
	for (int off = 1; off < 1024; off <<= 1) {
		const unsigned v = t >= off ? part[t - off] : 0u;
		__syncthreads();
		part[t] += v;
		__syncthreads();
	}
	unsigned run = part[t] - sum; // exclusive prefix of this thread's bins
	for (int j = 0; j < kPer; j++) {
		const unsigned c = dv.bins[t * kPer + j];
		dv.bins[t * kPer + j] = run;
		run += c;
	}
}
__global__ void k_shade_scatter(DeferView dv) {
	const long n = *dv.list_count;
	for (long e = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
	     e += static_cast<long>(gridDim.x) * blockDim.x) {
		const unsigned pos = atomicAdd(dv.bins + dv.key[e], 1u);
		if (kBoundsCheck && pos >= n)
			continue; // the slot left unwritten reads -1 in k_ref_shadow
		dv.sorted[pos] = static_cast<int>(e);
	}
}

__global__ void __launch_bounds__(128) k_ref_shadow(SceneView sv, const RefParams *__restrict__ params, DeferView dv,
                                                    int *status) {
	const RefParams &p = *params;
	Ctx c{sv, nullptr, &p, 0};
	const long total = static_cast<long>(*dv.list_count) * dv.taps;
	for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
	     i += static_cast<long>(gridDim.x) * blockDim.x) {
		const long slot = i / dv.taps;
		int k = static_cast<int>(i - slot * dv.taps);
		const long e = dv.sorted[slot];
		if (kBoundsCheck && (e < 0 || e >= dv.cap)) {
			c.err = 1;
			continue;
		}
		int l = 0;
		for (int n = vis_tap_count(p.lights[0]); k >= n; n = vis_tap_count(p.lights[l])) {
			k -= n;
			l++;
		}
		const size_t ri = static_cast<size_t>(dv.list[e]);
		const float4 r0 = dv.rec[3 * ri], r1 = dv.rec[3 * ri + 1];
		const V3 point = mk(r0.x, r0.y, r0.z);
		const VisTaps T = vis_taps(p.lights[l], point);
		// At a diffuse level, directLight multiplies this light's visibility by its
		// cone and incidence terms (direct_light_recorded, the same expressions): where
		// either is zero the light adds vis * 0 whatever the visibility, so its taps
		// need no ray. On the 1.31M-triangle 1080p x 2 spp frame this took the frame
		// from 35.2 to 31.1 ms with a bit-identical canvas (points on the lower half
		// of the sphere face away from the default light).
		bool needed = true;
		const int kind = __float_as_int(r0.w);
		if (kind == kLvDiffuse || kind == kLvDiffuseEnd) {
			const RefLight &L = p.lights[l];
			V3 ld;
			float atten;
			light_dir(L, point, ld, atten);
			float cone = 1.0f;
			if (L.type == kLightSpot)
				cone = (dot(-ld, normalize(l3(L.direction))) > L.cone_cos) ? 1.0f : 0.0f;
			const float incidence = smax(0.0f, dot(mk(r1.x, r1.y, r1.z), ld));
			needed = cone != 0.0f && incidence != 0.0f;
		}
		uint8_t occ = 0;
		if (!T.all_visible && needed) {
			V3 dir;
			float dist;
			vis_tap(T, point, k, dir, dist);
			occ = occluded(c, point, dir, dist, __float_as_int(r1.w)) ? 1 : 0;
		}
		dv.occl[e * dv.taps + (i - slot * dv.taps)] = occ;
	}
	if (c.err)
		atomicOr(status, 1);
}

__device__ __forceinline__ int unoccluded(const uint8_t *occ, int n) {
	int u = 0;
	for (int k = 0; k < n; k++)
		u += occ[k] ? 0 : 1;
	return u;
}

// directLight (src/Renderer.cpp:791-814) with each light's visibility counted from
// the recorded taps.
__device__ V3 direct_light_recorded(const RefParams &p, V3 point, V3 normal, V3 albedo, const uint8_t *occ) {
	V3 sum = mk(0, 0, 0);
	for (int li = 0; li < p.num_lights; li++) {
		const RefLight &L = p.lights[li];
		V3 ld;
		float atten;
		light_dir(L, point, ld, atten);
		float cone = 1.0f;
		if (L.type == kLightSpot)
			cone = (dot(-ld, normalize(l3(L.direction))) > L.cone_cos) ? 1.0f : 0.0f;
		const int n = vis_tap_count(L);
		const float vis = vis_fraction(unoccluded(occ, n), n);
		occ += n;
		const float incidence = smax(0.0f, dot(normal, ld));
		sum = sum + l3(L.colour) * (vis * cone * atten * incidence);
	}
	return albedo * vmin(sum, mk(1.0f, 1.0f, 1.0f));
}

// The subsurface branch's direct term (src/Renderer.cpp:857-880) with recorded visibility.
__device__ V3 subsurface_recorded(Ctx &c, V3 point, V3 n, V3 albedo, int ignore, const uint8_t *occ) {
	V3 shade = mk(0, 0, 0);
	const float wrap = 0.5f;
	for (int li = 0; li < c.p->num_lights; li++) {
		const RefLight &L = c.p->lights[li];
		const V3 to = l3(L.position) - point;
		const float dist = length(to);
		const V3 ld = to / dist;
		const float atten = L.intensity / (L.atten_constant + L.atten_linear * dist + L.atten_quadratic * dist * dist);
		const float wrap_diff = smax(0.0f, (dot(n, ld) + wrap) / (1.0f + wrap));
		const int nt = vis_tap_count(L);
		const float vis = vis_fraction(unoccluded(occ, nt), nt);
		occ += nt;
		shade = shade + albedo * l3(L.colour) * (vis * atten * wrap_diff);
		const Hit ex = intersect(c, point - n * 1e-3f, ld, ignore);
		const float thickness = ex.hit ? ex.t : 0.0f;
		shade = shade + albedo * l3(L.colour) * (atten * lm_exp(-3.0f * thickness) * 0.6f);
	}
	return vmin(shade, mk(1.5f, 1.5f, 1.5f));
}

__global__ void __launch_bounds__(128) k_ref_fold(SceneView sv, const float4 *__restrict__ ref_shade,
                                                  const RefParams *__restrict__ params, DeferView dv,
                                                  uint32_t *__restrict__ argb, float *__restrict__ mean_rgb,
                                                  int *status) {
	const RefParams &p = *params;
	const long li = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (li >= dv.npix)
		return;
	Ctx c{sv, ref_shade, &p, 0};
	V3 sum = mk(0, 0, 0);
	for (int s = 0; s < p.samples; s++) {
		const float4 *rec = dv.rec + 3 * ((static_cast<size_t>(li) * p.samples + s) * dv.levels);
		int last = 0;
		while (__float_as_int(rec[3 * last].w) < kLvDiffuseEnd)
			last++;
		V3 result = mk(0, 0, 0);
		for (int k = last; k >= 0; k--) {
			const float4 r0 = rec[3 * k], r1 = rec[3 * k + 1], r2 = rec[3 * k + 2];
			const int kind = __float_as_int(r0.w);
			const V3 b = mk(r2.x, r2.y, r2.z);
			if (kind == kLvValue) {
				result = b;
			} else if (kind == kLvMul) {
				result = b * result;
			} else if (kind != kLvPass) {
				const V3 point = mk(r0.x, r0.y, r0.z), n = mk(r1.x, r1.y, r1.z);
				const uint8_t *occ = dv.occl + static_cast<size_t>(__float_as_int(r2.w)) * dv.taps;
				const V3 direct = (kind == kLvSub || kind == kLvSubEnd)
				                      ? subsurface_recorded(c, point, n, b, __float_as_int(r1.w), occ)
				                      : direct_light_recorded(p, point, n, b, occ);
				result = (kind == kLvDiffuseEnd || kind == kLvSubEnd) ? direct : direct + b * result;
			}
		}
		sum = sum + result;
	}
	store_pixel(dv.pix0 + li, sum, p.samples, argb, mean_rgb);
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

size_t ref_defer_bytes_per_pixel(const RefParams &p) {
	int taps = 0;
	for (int i = 0; i < p.num_lights; i++)
		taps += ref_tap_count(p.lights[i]);
	const size_t records = static_cast<size_t>(std::max(p.samples, 0)) * (p.max_depth + 1);
	return records * (48 + 4 + 2 + 4 + static_cast<size_t>(taps));
}

cudaError_t launch_render_reference(const SceneView &sv, const float4 *ref_shade, const RefParams &p,
                                    const RefParams *d_params, uint32_t *argb, float *mean_rgb, int *status,
                                    void *scratch, size_t scratch_bytes, cudaStream_t st) {
	const long n = static_cast<long>(p.width) * p.height;
	if (n <= 0)
		return cudaSuccess;
	int taps = 0;
	for (int i = 0; i < p.num_lights; i++)
		taps += ref_tap_count(p.lights[i]);
	// samples <= 0 records nothing; the fold then writes the reference's 0 / samples.
	const size_t records = static_cast<size_t>(std::max(p.samples, 0)) * (p.max_depth + 1);
	const size_t per_pixel = ref_defer_bytes_per_pixel(p);
	const long fit = per_pixel == 0 ? n : static_cast<long>((scratch_bytes - kRefDeferFixedBytes) / per_pixel);
	const long chunk = std::max<long>(1, std::min<long>(n, fit));
	char *base = static_cast<char *>(scratch);
	DeferView dv;
	dv.list_count = reinterpret_cast<unsigned *>(base);
	dv.pix_next = dv.list_count + 1;
	base += 256;
	dv.bins = reinterpret_cast<unsigned *>(base);
	base += sizeof(unsigned) << kShadeKeyBits;
	dv.rec = reinterpret_cast<float4 *>(base);
	base += (static_cast<size_t>(chunk) * records * 48 + 255) & ~size_t(255);
	dv.list = reinterpret_cast<int *>(base);
	base += (static_cast<size_t>(chunk) * records * 4 + 255) & ~size_t(255);
	dv.key = reinterpret_cast<uint16_t *>(base);
	base += (static_cast<size_t>(chunk) * records * 2 + 255) & ~size_t(255);
	dv.sorted = reinterpret_cast<int *>(base);
	base += (static_cast<size_t>(chunk) * records * 4 + 255) & ~size_t(255);
	dv.occl = reinterpret_cast<uint8_t *>(base);
	dv.levels = p.max_depth + 1;
	dv.taps = taps;
	dv.cap = chunk * static_cast<long>(records);
	const int bs = 128;
	for (long p0 = 0; p0 < n; p0 += chunk) {
		dv.pix0 = p0;
		dv.npix = std::min(chunk, n - p0);
		cudaError_t e = cudaMemsetAsync(dv.list_count, 0, 2 * sizeof(unsigned), st);
		if (e != cudaSuccess)
			return e;
		e = cudaMemsetAsync(dv.bins, 0, sizeof(unsigned) << kShadeKeyBits, st);
		if (e != cudaSuccess)
			return e;
		{
			TraceRange r("paths");
			k_ref_paths<<<std::min(ceil_div(dv.npix, bs), 148 * 8), bs, 0, st>>>(sv, ref_shade, d_params, dv,
			                                                                   status);
		}
		if (kBoundsCheck) {
			// unwritten sort slots then read as -1, which k_ref_shadow reports
			e = cudaMemsetAsync(dv.sorted, 0xFF, static_cast<size_t>(dv.cap) * sizeof(int), st);
			if (e != cudaSuccess)
				return e;
		}
		k_shade_count<<<148 * 8, 256, 0, st>>>(dv);
		k_shade_scan<<<1, 1024, 0, st>>>(dv);
		k_shade_scatter<<<148 * 8, 256, 0, st>>>(dv);
		{
			TraceRange r("shadow rays");
			k_ref_shadow<<<148 * 16, bs, 0, st>>>(sv, d_params, dv, status);
		}
		TraceRange r("fold");
		k_ref_fold<<<ceil_div(dv.npix, bs), bs, 0, st>>>(sv, ref_shade, d_params, dv, argb, mean_rgb, status);
	}
	return cudaGetLastError();
}

} // namespace rnb
