// Photon mapping with reference semantics (renderPhotonMapped, src/Renderer.cpp:1177-1349;
// PhotonMap, src/Photon.cpp).
//
// Pass 1 of the reference traces numPhotons photons one after another from ONE
// std::mt19937(777) stream: a photon draws 2 numbers for its direction and then a
// path-dependent number more (a Fresnel choice at glass, a roulette draw and a
// cosine direction at diffuse surfaces), so photon i starts where photon i-1's
// draws ended. The GPU reproduces that sequence exactly, in parallel:
//   1. the engine's first M outputs are generated on the host (M bounds the total);
//   2. for EVERY position p < M a thread traces the photon that would start at p
//      and records how many draws it takes, c(p), and how many photons it deposits;
//   3. the chain s_0 = 0, s_{i+1} = s_i + c(s_i) is resolved by pointer doubling
//      (jump tables next^(2^k)), giving each photon its start;
//   4. deposit offsets are an exclusive scan over the chain, and the photons are
//      traced again from their starts, writing deposits at the reference's indices.
// The uniform grid of cells of side `radius` becomes a stable sort of the deposits
// by cell key, so a gather visits each cell's photons in insertion order and sums
// them in the reference's order. Pass 2 shades every pixel (mirror, metal and
// glass recursion on an explicit stack, direct light plus gathered irradiance at
// diffuse hits); with final gather, each image row consumes its own
// std::mt19937(1000 + y) stream in pixel order, one thread per row.
//
// Compiled with -fmad=false, like the other reference-semantics renderers.
#include <cub/cub.cuh>

#include <algorithm>
#include <random>
#include <vector>

#include "photon.hpp"
#include "refshade.cuh"

namespace rnb {

namespace {

constexpr int kPhotonDepth = 5;
constexpr int kMaxDrawsPerPhoton = 2 + 3 * (kPhotonDepth + 1);
constexpr int kMaxDepositsPerPhoton = kPhotonDepth + 1;
constexpr float kEmitScale = 1.8f;

struct PhotonInput {
	SceneView sv;
	const float4 *ref_shade;
	const uint32_t *draws;
	V3 origin;
	V3 power;
};

// tracePhoton (src/Renderer.cpp:1177-1235), iteratively (each call recurses at most
// once, at its end). Reads the engine outputs from draws[p...]; returns the number
// of draws taken. With out != nullptr the deposits are written there.
__device__ int trace_photon(const PhotonInput &in, uint32_t p0, float4 *out_pos, float4 *out_pow, float4 *out_dir,
                            int out_room, int &deposits, int &err) {
	uint32_t p = p0;
	auto U = [&]() { return canonical01(in.draws[p++]); };
	const float z = 1.0f - 2.0f * U();
	const float a = 2.0f * 3.14159265f * U();
	const float r = sqrtf(smax(0.0f, 1.0f - z * z));
	V3 origin = in.origin;
	V3 direction = mk(r * lm_cos(a), z, r * lm_sin(a));
	V3 power = in.power;
	deposits = 0;
	for (int depth = kPhotonDepth; depth >= 0; depth--) {
		const RayPre ray = make_ray(origin.x, origin.y, origin.z, direction.x, direction.y, direction.z);
		const HitRec h = trace_closest_best<kOrderReference>(in.sv, ray, -1, err);
		if (h.idx < 0)
			break;
		const float4 s0 = in.ref_shade[2 * h.idx], s1 = in.ref_shade[2 * h.idx + 1];
		const int mat = __float_as_int(s0.w);
		const V3 tri_n = mk(s0.x, s0.y, s0.z);
		const V3 point = origin + h.t * direction;
		const V3 n = face_viewer(tri_n, direction);
		if (mat == kRefMirror) {
			const V3 rr = reflect(direction, n);
			origin = point + 1e-4f * rr;
			direction = rr;
			continue;
		}
		if (mat == kRefMetal) {
			const V3 albedo = base_colour(mat, mk(s1.x, s1.y, s1.z), point) / 255.0f;
			const V3 rr = reflect(direction, n);
			origin = point + 1e-4f * rr;
			direction = rr;
			power = power * albedo;
			continue;
		}
		if (mat == kRefGlass) {
			const float ior = 1.5f;
			V3 nn = tri_n;
			float cosi = dot(direction, nn);
			float etai = 1.0f, etat = ior;
			if (cosi < 0.0f) {
				cosi = -cosi;
			} else {
				const float tmp = etai;
				etai = etat;
				etat = tmp;
				nn = -nn;
			}
			float r0 = (etai - etat) / (etai + etat);
			r0 *= r0;
			const float fresnel = r0 + (1.0f - r0) * lm_pow(1.0f - cosi, 5.0f);
			const V3 refr = refract(direction, nn, etai / etat);
			const V3 d = (length(refr) < 1e-6f || U() < fresnel) ? reflect(direction, nn) : refr;
			origin = point + 1e-4f * d;
			direction = d;
			continue;
		}
		// deposit on the diffuse surface, then maybe bounce (roulette by albedo)
		if (out_pos) {
			if (kBoundsCheck && deposits >= out_room) {
				err = 1;
				break;
			}
			out_pos[deposits] = make_float4(point.x, point.y, point.z, 0.0f);
			out_pow[deposits] = make_float4(power.x, power.y, power.z, 0.0f);
			out_dir[deposits] = make_float4(direction.x, direction.y, direction.z, 0.0f);
		}
		deposits++;
		const V3 albedo = base_colour(mat, mk(s1.x, s1.y, s1.z), point) / 255.0f;
		// std::max({r, g, b}): the first largest
		float pmax = albedo.x;
		if (pmax < albedo.y)
			pmax = albedo.y;
		if (pmax < albedo.z)
			pmax = albedo.z;
		if (!(depth > 0 && U() < pmax))
			break;
		const float u1 = U();
		const float u2 = U();
		const V3 d = cosine_hemisphere_u(n, u1, u2);
		origin = point + 1e-4f * d;
		direction = d;
		power = power * albedo / pmax;
	}
	return static_cast<int>(p - p0);
}

__global__ void __launch_bounds__(128) k_photon_counts(PhotonInput in, uint32_t n_pos, uint32_t *next,
                                                       uint8_t *deposits, int *status) {
	const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n_pos)
		return;
	int err = 0, d = 0;
	const int c = trace_photon(in, p, nullptr, nullptr, nullptr, 0, d, err);
	next[p] = p + static_cast<uint32_t>(c);
	deposits[p] = static_cast<uint8_t>(d);
	if (err)
		atomicOr(status, 1);
}

// jump_out[p] = jump_in[jump_in[p]] (positions past the table stay put).
__global__ void k_jump_square(const uint32_t *__restrict__ jin, uint32_t *__restrict__ jout, uint32_t n_pos) {
	const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n_pos)
		return;
	const uint32_t q = jin[p];
	jout[p] = q < n_pos ? jin[q] : q;
}

// start[i] = next^i(0), from the binary digits of i.
__global__ void k_chain_starts(const uint32_t *__restrict__ jumps, uint32_t n_pos, int levels, uint32_t n_photons,
                               const uint8_t *__restrict__ deposits, uint32_t *__restrict__ start,
                               uint32_t *__restrict__ count) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n_photons)
		return;
	uint32_t pos = 0;
	for (int k = 0; k < levels && pos < n_pos; k++)
		if ((i >> k) & 1u)
			pos = jumps[static_cast<size_t>(k) * n_pos + pos];
	start[i] = pos;
	count[i] = pos < n_pos ? deposits[pos] : 0u;
}

__global__ void __launch_bounds__(128) k_photon_deposit(PhotonInput in, uint32_t n_photons,
                                                        const uint32_t *__restrict__ start,
                                                        const uint32_t *__restrict__ offset, float4 *pos,
                                                        float4 *pw, float4 *dir, uint32_t cap, int *status) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n_photons)
		return;
	int err = 0, d = 0;
	const uint32_t o = offset[i];
	trace_photon(in, start[i], pos + o, pw + o, dir + o, o < cap ? static_cast<int>(cap - o) : 0, d, err);
	if (err)
		atomicOr(status, 1);
}

// PhotonMap::cellKey / build (src/Photon.cpp:5-19).
__device__ __forceinline__ long long cell_key(int x, int y, int z) {
	auto f = [](int v) -> long long { return static_cast<long long>((v + (1 << 20)) & 0x1FFFFF); };
	return (f(x) << 42) | (f(y) << 21) | f(z);
}
__device__ __forceinline__ int cell_coord(float v, float cell) { return static_cast<int>(floorf(v / cell)); }

__global__ void k_photon_keys(const float4 *__restrict__ pos, uint32_t n, float cell,
                              unsigned long long *__restrict__ keys, uint32_t *__restrict__ idx) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const float4 p = pos[i];
	keys[i] = static_cast<unsigned long long>(
	    cell_key(cell_coord(p.x, cell), cell_coord(p.y, cell), cell_coord(p.z, cell)));
	idx[i] = i;
}

struct PhotonMapView {
	const unsigned long long *keys; // sorted cell keys
	const uint32_t *idx;            // photon index of each sorted entry (ascending within a cell)
	const float4 *pos, *pw, *dir;
	uint32_t n;
	float cell;
	float radius;
};

// PhotonMap::gather (src/Photon.cpp:21-46): the 27 cells in the reference's loop
// order, each cell's photons in insertion order.
__device__ V3 gather(const PhotonMapView &m, V3 point, V3 normal) {
	const int cx = cell_coord(point.x, m.cell), cy = cell_coord(point.y, m.cell), cz = cell_coord(point.z, m.cell);
	V3 sum = mk(0.0f, 0.0f, 0.0f);
	const float r2 = m.radius * m.radius;
	for (int dx = -1; dx <= 1; dx++)
		for (int dy = -1; dy <= 1; dy++)
			for (int dz = -1; dz <= 1; dz++) {
				const unsigned long long key = static_cast<unsigned long long>(cell_key(cx + dx, cy + dy, cz + dz));
				uint32_t lo = 0, hi = m.n;
				while (lo < hi) {
					const uint32_t mid = (lo + hi) >> 1;
					if (m.keys[mid] < key)
						lo = mid + 1;
					else
						hi = mid;
				}
				for (uint32_t e = lo; e < m.n && m.keys[e] == key; e++) {
					const uint32_t pi = m.idx[e];
					const float4 pp = m.pos[pi];
					const V3 d = mk(pp.x, pp.y, pp.z) - point;
					if (dot(d, d) > r2)
						continue;
					const float4 pd = m.dir[pi];
					if (dot(normal, -mk(pd.x, pd.y, pd.z)) <= 0.0f)
						continue;
					const float4 pw = m.pw[pi];
					sum = sum + mk(pw.x, pw.y, pw.z);
				}
			}
	return sum / (3.14159265f * r2);
}

// photonShade (src/Renderer.cpp:1242-1298) on an explicit stack: mirror and metal
// frames take one child, glass frames a reflection and (unless totally reflected)
// a refraction, combined as the reference combines them.
struct PFrame {
	V3 co[2], cd[2], res[2];
	V3 tint;
	float fres;
	int n, next, kind, tir, depth;
};
constexpr int kPMirror = 0, kPMetal = 1, kPGlass = 2;
constexpr int kPhotonShadeDepth = 4;

// Shading of a diffuse hit; with gather_rays > 0 the final gather draws from rng.
__device__ V3 photon_diffuse(Ctx &c, const PhotonMapView &m, int idx, V3 point, V3 n, V3 albedo, int gather_rays,
                             MT *rng) {
	const V3 direct = direct_light(c, point, n, albedo, idx);
	V3 indirect;
	if (gather_rays > 0) {
		V3 gathered = mk(0.0f, 0.0f, 0.0f);
		for (int i = 0; i < gather_rays; i++) {
			const V3 gdir = cosine_hemisphere(n, *rng);
			const Hit gh = intersect(c, point + 1e-4f * gdir, gdir, -1);
			if (gh.hit) {
				const float4 g0 = c.ref_shade[2 * gh.idx];
				gathered = gathered + gather(m, gh.point, face_viewer(mk(g0.x, g0.y, g0.z), gdir));
			} else {
				gathered = gathered + environment(gdir) / 255.0f;
			}
		}
		indirect = albedo * gathered / static_cast<float>(gather_rays);
	} else {
		indirect = albedo * gather(m, point, n);
	}
	return direct + indirect;
}

__device__ bool photon_expand(Ctx &c, const PhotonMapView &m, V3 o, V3 d, int depth, int gather_rays, MT *rng,
                              V3 &value, PFrame &f) {
	const Hit hit = intersect(c, o, d, -1);
	if (!hit.hit) {
		value = environment(d) / 255.0f;
		return true;
	}
	const float4 s0 = c.ref_shade[2 * hit.idx], s1 = c.ref_shade[2 * hit.idx + 1];
	const int mat = __float_as_int(s0.w);
	const V3 tri_n = mk(s0.x, s0.y, s0.z);
	const V3 point = hit.point;
	const V3 n = face_viewer(tri_n, d);
	f.depth = depth;
	f.next = 0;
	f.tir = 0;
	if (depth > 0 && (mat == kRefMirror || mat == kRefMetal)) {
		const V3 r = reflect(d, n);
		f.co[0] = point + 1e-4f * r;
		f.cd[0] = r;
		f.n = 1;
		f.kind = mat == kRefMirror ? kPMirror : kPMetal;
		f.tint = base_colour(mat, mk(s1.x, s1.y, s1.z), point) / 255.0f;
		return false;
	}
	if (depth > 0 && mat == kRefGlass) {
		V3 nn = tri_n;
		float cosi = dot(d, nn);
		float etai = 1.0f, etat = 1.5f;
		if (cosi < 0.0f) {
			cosi = -cosi;
		} else {
			const float tmp = etai;
			etai = etat;
			etat = tmp;
			nn = -nn;
		}
		float r0 = (etai - etat) / (etai + etat);
		r0 *= r0;
		f.fres = r0 + (1.0f - r0) * lm_pow(1.0f - cosi, 5.0f);
		const V3 refl = reflect(d, nn);
		f.co[0] = point + 1e-4f * refl;
		f.cd[0] = refl;
		const V3 refr = refract(d, nn, etai / etat);
		f.kind = kPGlass;
		f.n = 2;
		if (length(refr) < 1e-6f) {
			f.tir = 1;
			f.n = 1;
		} else {
			f.co[1] = point + 1e-4f * refr;
			f.cd[1] = refr;
		}
		return false;
	}
	const V3 albedo = base_colour(mat, mk(s1.x, s1.y, s1.z), point) / 255.0f;
	value = photon_diffuse(c, m, hit.idx, point, n, albedo, gather_rays, rng);
	return true;
}

__device__ V3 photon_shade(Ctx &c, const PhotonMapView &m, V3 o, V3 d, int gather_rays, MT *rng) {
	PFrame st[kPhotonShadeDepth + 1];
	V3 v;
	if (photon_expand(c, m, o, d, kPhotonShadeDepth, gather_rays, rng, v, st[0]))
		return v;
	int sp = 1;
	for (;;) {
		PFrame &f = st[sp - 1];
		if (f.next < f.n) {
			const int i = f.next;
			if (photon_expand(c, m, f.co[i], f.cd[i], f.depth - 1, gather_rays, rng, v, st[sp])) {
				f.res[i] = v;
				f.next++;
			} else {
				sp++;
			}
			continue;
		}
		if (f.kind == kPMirror)
			v = f.res[0];
		else if (f.kind == kPMetal)
			v = f.tint * f.res[0];
		else
			v = f.tir ? f.res[0] : f.fres * f.res[0] + (1.0f - f.fres) * f.res[1];
		if (--sp == 0)
			return v;
		PFrame &parent = st[sp - 1];
		parent.res[parent.next] = v;
		parent.next++;
	}
}

__device__ uint32_t pack_pixel(V3 colour) {
	const int r = min(255, cvt_trunc(colour.x));
	const int g = min(255, cvt_trunc(colour.y));
	const int b = min(255, cvt_trunc(colour.z));
	return (255u << 24) | ((static_cast<uint32_t>(r) & 0xFFu) << 16) | ((static_cast<uint32_t>(g) & 0xFFu) << 8) |
	       (static_cast<uint32_t>(b) & 0xFFu);
}

// Camera ray of pixel (x, y) as renderPhotonMapped forms it (src/Renderer.cpp:1331-1333).
__device__ V3 photon_camera_dir(const RefParams &p, int x, int y) {
	const V3 right = mk(p.orient[0], p.orient[1], p.orient[2]);
	const V3 upv = mk(p.orient[3], p.orient[4], p.orient[5]);
	const V3 fwd = mk(p.orient[6], p.orient[7], p.orient[8]);
	const V3 dc = mk((static_cast<float>(x) - static_cast<float>(p.width) / 2.0f) / p.f,
	                 -(static_cast<float>(y) - static_cast<float>(p.height) / 2.0f) / p.f, -1.0f);
	return normalize(right * dc.x + upv * dc.y + fwd * dc.z);
}

__global__ void __launch_bounds__(128) k_photon_pixels(SceneView sv, const float4 *__restrict__ ref_shade,
                                                       const RefParams *__restrict__ params, PhotonMapView m,
                                                       uint32_t *__restrict__ argb, int *status) {
	const RefParams &p = *params;
	const long pix = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (pix >= static_cast<long>(p.width) * p.height)
		return;
	const int x = static_cast<int>(pix % p.width), y = static_cast<int>(pix / p.width);
	Ctx c{sv, ref_shade, &p, 0};
	const V3 colour = photon_shade(c, m, l3(p.position), photon_camera_dir(p, x, y), 0, nullptr) * 255.0f;
	argb[pix] = pack_pixel(colour);
	if (c.err)
		atomicOr(status, 1);
}

// Final gather: row y draws from std::mt19937(1000 + y) in pixel order.
__global__ void __launch_bounds__(64) k_photon_rows(SceneView sv, const float4 *__restrict__ ref_shade,
                                                    const RefParams *__restrict__ params, PhotonMapView m,
                                                    int gather_rays, uint32_t *__restrict__ argb, int *status) {
	const RefParams &p = *params;
	const int y = blockIdx.x * blockDim.x + threadIdx.x;
	if (y >= p.height)
		return;
	Ctx c{sv, ref_shade, &p, 0};
	MT rng;
	rng.seed(1000u + static_cast<uint32_t>(y));
	for (int x = 0; x < p.width; x++) {
		const V3 colour = photon_shade(c, m, l3(p.position), photon_camera_dir(p, x, y), gather_rays, &rng) * 255.0f;
		argb[static_cast<size_t>(y) * p.width + x] = pack_pixel(colour);
	}
	if (c.err)
		atomicOr(status, 1);
}

inline size_t align256(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }

} // namespace

cudaError_t photon_scratch_bytes(int n_photons, size_t &bytes) {
	const size_t n_pos = static_cast<size_t>(n_photons) * kMaxDrawsPerPhoton + 8;
	const size_t n_draws = n_pos + kMaxDrawsPerPhoton + 8;
	int levels = 1;
	while ((1ull << levels) < static_cast<unsigned long long>(n_photons))
		levels++;
	const size_t n_dep = static_cast<size_t>(n_photons) * kMaxDepositsPerPhoton;
	size_t cub_bytes = 0, scan_bytes = 0;
	cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, static_cast<unsigned long long *>(nullptr),
	                                                static_cast<unsigned long long *>(nullptr),
	                                                static_cast<uint32_t *>(nullptr),
	                                                static_cast<uint32_t *>(nullptr), static_cast<int>(n_dep));
	if (e != cudaSuccess)
		return e;
	e = cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, static_cast<uint32_t *>(nullptr),
	                                  static_cast<uint32_t *>(nullptr), n_photons + 1);
	if (e != cudaSuccess)
		return e;
	bytes = align256(n_draws * 4) + align256(n_pos * 4) * static_cast<size_t>(levels) + align256(n_pos) +
	        3 * align256((static_cast<size_t>(n_photons) + 1) * 4) + 3 * align256(n_dep * 16) +
	        2 * align256(n_dep * 8) + 2 * align256(n_dep * 4) + align256(std::max(cub_bytes, scan_bytes)) + 1024;
	return cudaSuccess;
}

cudaError_t launch_photon_mapped(const SceneView &sv, const float4 *ref_shade, const RefParams &hp,
                                 const RefParams *d_params, int n_photons, int gather_rays, void *scratch,
                                 size_t scratch_bytes, uint32_t *argb, int *status, cudaStream_t st,
                                 unsigned *deposits_out) {
	const size_t n_pos = static_cast<size_t>(n_photons) * kMaxDrawsPerPhoton + 8;
	const size_t n_draws = n_pos + kMaxDrawsPerPhoton + 8;
	int levels = 1;
	while ((1ull << levels) < static_cast<unsigned long long>(n_photons))
		levels++;
	const size_t n_dep = static_cast<size_t>(n_photons) * kMaxDepositsPerPhoton;
	// carve the scratch
	char *b = static_cast<char *>(scratch);
	auto take = [&b](size_t bytes) {
		char *p = b;
		b += align256(bytes);
		return p;
	};
	uint32_t *d_draws = reinterpret_cast<uint32_t *>(take(n_draws * 4));
	uint32_t *d_jumps = reinterpret_cast<uint32_t *>(take(n_pos * 4 * static_cast<size_t>(levels)));
	uint8_t *d_dep = reinterpret_cast<uint8_t *>(take(n_pos));
	uint32_t *d_start = reinterpret_cast<uint32_t *>(take((static_cast<size_t>(n_photons) + 1) * 4));
	uint32_t *d_count = reinterpret_cast<uint32_t *>(take((static_cast<size_t>(n_photons) + 1) * 4));
	uint32_t *d_off = reinterpret_cast<uint32_t *>(take((static_cast<size_t>(n_photons) + 1) * 4));
	float4 *d_pos = reinterpret_cast<float4 *>(take(n_dep * 16));
	float4 *d_pw = reinterpret_cast<float4 *>(take(n_dep * 16));
	float4 *d_dir = reinterpret_cast<float4 *>(take(n_dep * 16));
	unsigned long long *d_k0 = reinterpret_cast<unsigned long long *>(take(n_dep * 8));
	unsigned long long *d_k1 = reinterpret_cast<unsigned long long *>(take(n_dep * 8));
	uint32_t *d_i0 = reinterpret_cast<uint32_t *>(take(n_dep * 4));
	uint32_t *d_i1 = reinterpret_cast<uint32_t *>(take(n_dep * 4));
	void *d_tmp = take(0);
	const size_t used = static_cast<size_t>(b - static_cast<char *>(scratch));
	if (used > scratch_bytes)
		return cudaErrorInvalidValue;
	const size_t tmp_bytes = scratch_bytes - used;

	// 1. the engine's outputs: std::mt19937(777), as the reference seeds it
	std::vector<uint32_t> draws(n_draws);
	std::mt19937 gen(777u);
	for (size_t i = 0; i < n_draws; i++)
		draws[i] = static_cast<uint32_t>(gen());
	cudaError_t e = cudaMemcpyAsync(d_draws, draws.data(), n_draws * 4, cudaMemcpyHostToDevice, st);
	if (e != cudaSuccess)
		return e;
	// the emitting light: the first light (src/Renderer.cpp:1315-1323)
	const RefLight &L = hp.lights[0];
	PhotonInput in;
	in.sv = sv;
	in.ref_shade = ref_shade;
	in.draws = d_draws;
	in.origin = V3{L.position[0], L.position[1], L.position[2]};
	const float scale = L.intensity * kEmitScale / static_cast<float>(n_photons);
	in.power = V3{L.colour[0] * scale, L.colour[1] * scale, L.colour[2] * scale};

	// 2. draws and deposits of a photon starting at every position
	const int bs = 128;
	k_photon_counts<<<ceil_div(static_cast<long>(n_pos), bs), bs, 0, st>>>(in, static_cast<uint32_t>(n_pos), d_jumps,
	                                                                        d_dep, status);
	// 3. jump tables next^(2^k), then every photon's start
	for (int k = 1; k < levels; k++)
		k_jump_square<<<ceil_div(static_cast<long>(n_pos), 256), 256, 0, st>>>(
		    d_jumps + static_cast<size_t>(k - 1) * n_pos, d_jumps + static_cast<size_t>(k) * n_pos,
		    static_cast<uint32_t>(n_pos));
	k_chain_starts<<<ceil_div(static_cast<long>(n_photons), 256), 256, 0, st>>>(
	    d_jumps, static_cast<uint32_t>(n_pos), levels, static_cast<uint32_t>(n_photons), d_dep, d_start, d_count);
	e = cudaMemsetAsync(d_count + n_photons, 0, 4, st);
	if (e != cudaSuccess)
		return e;
	// 4. deposit offsets, then the photons themselves
	size_t tb = tmp_bytes;
	e = cub::DeviceScan::ExclusiveSum(d_tmp, tb, d_count, d_off, n_photons + 1, st);
	if (e != cudaSuccess)
		return e;
	uint32_t n_total = 0;
	e = cudaMemcpyAsync(&n_total, d_off + n_photons, 4, cudaMemcpyDeviceToHost, st);
	if (e != cudaSuccess)
		return e;
	e = cudaStreamSynchronize(st);
	if (e != cudaSuccess)
		return e;
	if (deposits_out)
		*deposits_out = n_total;
	k_photon_deposit<<<ceil_div(static_cast<long>(n_photons), bs), bs, 0, st>>>(in, static_cast<uint32_t>(n_photons),
	                                                                            d_start, d_off, d_pos, d_pw, d_dir,
	                                                                            static_cast<uint32_t>(n_dep), status);
	// the grid: a stable sort of the deposits by cell key
	const float radius = 0.25f;
	PhotonMapView m{};
	m.pos = d_pos;
	m.pw = d_pw;
	m.dir = d_dir;
	m.n = n_total;
	m.cell = radius;
	m.radius = radius;
	if (n_total > 0) {
		k_photon_keys<<<ceil_div(static_cast<long>(n_total), 256), 256, 0, st>>>(d_pos, n_total, radius, d_k0, d_i0);
		tb = tmp_bytes;
		e = cub::DeviceRadixSort::SortPairs(d_tmp, tb, d_k0, d_k1, d_i0, d_i1, static_cast<int>(n_total), 0, 64, st);
		if (e != cudaSuccess)
			return e;
		m.keys = d_k1;
		m.idx = d_i1;
	} else {
		m.keys = d_k0;
		m.idx = d_i0;
	}
	// pass 2
	const long npix = static_cast<long>(hp.width) * hp.height;
	if (gather_rays > 0)
		k_photon_rows<<<ceil_div(static_cast<long>(hp.height), 64), 64, 0, st>>>(sv, ref_shade, d_params, m,
		                                                                         gather_rays, argb, status);
	else
		k_photon_pixels<<<ceil_div(npix, bs), bs, 0, st>>>(sv, ref_shade, d_params, m, argb, status);
	return cudaGetLastError();
}

} // namespace rnb
