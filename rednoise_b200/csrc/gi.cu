// Bidirectional path tracing and primary-sample Metropolis light transport with
// reference semantics (src/BDPT.cpp:8-144, src/Metropolis.cpp:8-192): diffuse-only
// estimators lit by a fixed 0.36 x 0.36 emitter at (0, 0.33, 0) facing -y with
// Le = 30, four bounces, Reinhard tone mapping onto the 8-bit canvas.
//
// Bidirectional, reference stream: every image row draws from its own
// std::mt19937(9871 + y) in the reference's order, so the canvas equals the
// reference's. The number of draws a sample takes depends on its subpath lengths,
// so a row's samples are found in stream order: one thread per row traces the
// camera and light subpaths (the closest-hit chain) and records their vertices;
// then the connections (the shadow rays, most of the work) run one thread per
// connection and are summed per pixel in the reference's order. Columns are processed in chunks so
// the vertex records stay within a fixed budget; the row streams persist in
// device memory between chunks.
//
// Bidirectional, counter stream: the same estimator with each (pixel, sample)
// drawing from Philox-4x32-10 under the seed; the subpaths are traced one thread
// per sample, then the same connection passes.
//
// Metropolis: many chains run in parallel, one thread each. A bootstrap of
// independent paths estimates the normalisation b as the reference does; chain
// starts are drawn from the bootstrap paths with probability proportional to
// luminance (so every chain starts in the stationary distribution and short chains
// carry no start-up bias); each chain then applies the reference's mutations
// (large step with probability 0.3, else a Gaussian perturbation of sigma 0.02 on
// every coordinate, wrapped into [0, 1)), its acceptance rule and its expected-value
// deposits into the image. All random numbers come from Philox streams.
//
// This file is compiled with -fmad=false: expressions are separately rounded IEEE
// operations in source order, as in the reference's non-FMA x86-64 build.
#include <algorithm>

#include "gi.hpp"
#include "refshade.cuh"
#include "rng.cuh"
#include "trace_range.hpp"

namespace rnb {

namespace {

constexpr float kGiPi = 3.14159265f;
constexpr float kGiEps = 1e-3f;
constexpr float kGiLightHalf = 0.18f;
constexpr int kGiMaxDepth = 4;
constexpr int kMltDims = 2 + 4 * kGiMaxDepth;
constexpr int kRowsPerBlock = 1;

__device__ __forceinline__ float gi_light_area() { return (2.0f * kGiLightHalf) * (2.0f * kGiLightHalf); }

// std::mt19937 of one image row kept in device memory: 624 contiguous words, so
// the row's lone thread finds its state in a few cache lines.
struct MtRow {
	uint32_t *s;
	int i;
	__device__ void twist() {
		for (int k = 0; k < 624; k++) {
			const uint32_t y = (s[k] & 0x80000000u) | (s[k + 1 < 624 ? k + 1 : 0] & 0x7fffffffu);
			const int m = k + 397 < 624 ? k + 397 : k + 397 - 624;
			s[k] = s[m] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
		}
		i = 0;
	}
	__device__ float operator()() {
		if (i >= 624)
			twist();
		uint32_t y = s[i++];
		y ^= y >> 11;
		y ^= (y << 7) & 0x9d2c5680u;
		y ^= (y << 15) & 0xefc60000u;
		y ^= y >> 18;
		return canonical01(y);
	}
};

__device__ __forceinline__ uint32_t u4_word(U4 v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }

// Philox words of counter (a, b, block, tag) under the seed, consumed in order and
// mapped as the reference maps an engine output.
struct CtrDraw {
	uint32_t a, b, tag, k0, k1;
	int n;
	U4 blk;
	__device__ float operator()() {
		if ((n & 3) == 0)
			blk = philox4x32_10(U4{a, b, static_cast<uint32_t>(n >> 2), tag}, k0, k1);
		const int w = n & 3;
		n++;
		return canonical01(u4_word(blk, w));
	}
};

struct GV {
	V3 p, n, albedo, beta;
};

struct GiCam {
	V3 pos, right, up, fwd;
};

__device__ __forceinline__ GiCam gi_cam(const GiParams &p) {
	return {mk(p.position[0], p.position[1], p.position[2]), mk(p.orient[0], p.orient[1], p.orient[2]),
	        mk(p.orient[3], p.orient[4], p.orient[5]), mk(p.orient[6], p.orient[7], p.orient[8])};
}

__device__ __forceinline__ V3 tri_normal(const float4 *ref_shade, int idx) {
	const float4 s0 = __ldg(ref_shade + 2 * static_cast<size_t>(idx));
	return mk(s0.x, s0.y, s0.z);
}
// vec3(colour) / 255 (src/BDPT.cpp:38-40)
__device__ __forceinline__ V3 tri_albedo(const float4 *ref_shade, int idx) {
	const float4 s1 = __ldg(ref_shade + 2 * static_cast<size_t>(idx) + 1);
	return mk(s1.x, s1.y, s1.z) / 255.0f;
}

// Closest hit for a thread that runs alone (the row pass): the same result as
// intersect(), with each leaf's triangle tests overlapped.
__device__ __forceinline__ Hit intersect_alone(Ctx &c, V3 o, V3 d) {
	const RayPre r = make_ray(o.x, o.y, o.z, d.x, d.y, d.z);
	HitRec h;
	if (c.sv.nodes4 && finite_inverse(r)) {
		LocalStack<unsigned long long> st;
		h = trace_closest4_flat(c.sv, r, -1, c.err, st);
	} else {
		h = trace_closest<kOrderReference>(c.sv, r, -1, c.err);
	}
	Hit out;
	out.hit = h.idx >= 0;
	out.idx = h.idx;
	out.t = h.t;
	out.point = o + h.t * d;
	return out;
}

// tracePath (src/BDPT.cpp:43-61). code (may be null) receives 2 * triangle + 1 if
// faceViewer flipped the normal.
template <bool kAlone, class D>
__device__ int gi_subpath(Ctx &c, V3 o, V3 d, V3 beta, GV *out, int *code, D &draw) {
	int k = 0;
	for (int depth = 0; depth < kGiMaxDepth; depth++) {
		const Hit h = kAlone ? intersect_alone(c, o, d) : intersect(c, o, d, -1);
		if (!h.hit)
			break;
		const V3 tn = tri_normal(c.ref_shade, h.idx);
		const bool flip = !(dot(tn, d) < 0.0f); // faceViewer (src/BDPT.cpp:34-36)
		GV v;
		v.p = h.point;
		v.n = flip ? -tn : tn;
		v.albedo = tri_albedo(c.ref_shade, h.idx);
		v.beta = beta;
		out[k] = v;
		if (code)
			code[k] = 2 * h.idx + (flip ? 1 : 0);
		k++;
		const float u1 = draw(), u2 = draw();
		const V3 nd = cosine_hemisphere_u(v.n, u1, u2);
		beta = beta * v.albedo;
		o = v.p + kGiEps * nd;
		d = nd;
	}
	return k;
}

// The camera and light subpaths of one sample (src/BDPT.cpp:90-108). lv[0] is the
// point on the emitter; nl counts it.
template <bool kAlone, class D>
__device__ void bdpt_subpaths(Ctx &c, const GiParams &p, const GiCam &cam, int x, int y, D &draw, GV *cv, int *ccode,
                              int &nc, GV *lv, int *lcode, int &nl) {
	// glm::vec3((x + U - W/2) / f, -(y + U - H/2) / f, -1): GCC evaluates the two
	// random arguments right to left, so the y jitter is drawn first.
	const float uy = draw(), ux = draw();
	const float sx = (static_cast<float>(x) + ux - static_cast<float>(p.width) / 2.0f) / p.f;
	const float sy = -(static_cast<float>(y) + uy - static_cast<float>(p.height) / 2.0f) / p.f;
	const V3 dir = normalize(cam.right * sx + cam.up * sy + cam.fwd * -1.0f);
	nc = gi_subpath<kAlone>(c, cam.pos, dir, mk(1.0f, 1.0f, 1.0f), cv, ccode, draw);
	const float lz = draw(), lx = draw(); // right to left again
	const V3 lp =
	    mk(0.0f, 0.33f, 0.0f) + mk((lx * 2.0f - 1.0f) * kGiLightHalf, 0.0f, (lz * 2.0f - 1.0f) * kGiLightHalf);
	const V3 ln = mk(0.0f, -1.0f, 0.0f);
	const V3 le = mk(30.0f, 30.0f, 30.0f) * gi_light_area();
	lv[0] = GV{lp, ln, mk(0.0f, 0.0f, 0.0f), le};
	const float d1 = draw(), d2 = draw();
	const V3 ldir = cosine_hemisphere_u(ln, d1, d2);
	nl = 1 + gi_subpath<kAlone>(c, lp + kGiEps * ldir, ldir, le, lv + 1, lcode, draw);
}

// Reinhard and the 8-bit pack (src/BDPT.cpp:137-141, src/Metropolis.cpp:185-189).
__device__ __forceinline__ uint32_t gi_pack(V3 c) {
	c = 255.0f * mk(c.x / (c.x + 1.0f), c.y / (c.y + 1.0f), c.z / (c.z + 1.0f));
	const int r = min(255, cvt_trunc(c.x)), g = min(255, cvt_trunc(c.y)), b = min(255, cvt_trunc(c.z));
	return (255u << 24) | ((static_cast<uint32_t>(r) & 0xFFu) << 16) | ((static_cast<uint32_t>(g) & 0xFFu) << 8) |
	       (static_cast<uint32_t>(b) & 0xFFu);
}

__device__ __forceinline__ void gi_store(const GiParams &p, long pix, V3 col, uint32_t *argb, float *rgb) {
	argb[pix] = gi_pack(col);
	if (rgb) {
		rgb[3 * pix] = col.x;
		rgb[3 * pix + 1] = col.y;
		rgb[3 * pix + 2] = col.z;
	}
}

__global__ void k_mt_seed_rows(uint32_t *s, int *idx, int rows) {
	const int y = blockIdx.x * blockDim.x + threadIdx.x;
	if (y >= rows)
		return;
	uint32_t *row = s + 624 * static_cast<size_t>(y);
	uint32_t v = 9871u + static_cast<uint32_t>(y);
	row[0] = v;
	for (int k = 1; k < 624; k++) {
		v = 1812433253u * (v ^ (v >> 30)) + static_cast<uint32_t>(k);
		row[k] = v;
	}
	idx[y] = 624;
}

// Traces one sample's subpaths and records them: camera vertices in slots 0-3,
// the emitter point in slot 4, light vertices in slots 5-8 (16 B each: position
// and 2 * triangle + normal flip), and the two lengths in cnt.
template <bool kAlone, class D>
__device__ __forceinline__ void record_sample(Ctx &c, const GiParams &p, const GiCam &cam, int x, int y, D &draw,
                                              float4 *__restrict__ rec, uint8_t *__restrict__ cnt, size_t sample) {
	GV cv[kGiMaxDepth], lv[kGiMaxDepth + 1];
	int cc[kGiMaxDepth], lc[kGiMaxDepth], nc, nl;
	bdpt_subpaths<kAlone>(c, p, cam, x, y, draw, cv, cc, nc, lv, lc, nl);
	float4 *r = rec + sample * kBdptRecordSlots;
	for (int i = 0; i < nc; i++)
		r[i] = make_float4(cv[i].p.x, cv[i].p.y, cv[i].p.z, __int_as_float(cc[i]));
	r[kGiMaxDepth] = make_float4(lv[0].p.x, lv[0].p.y, lv[0].p.z, 0.0f);
	for (int j = 1; j < nl; j++)
		r[kGiMaxDepth + j] = make_float4(lv[j].p.x, lv[j].p.y, lv[j].p.z, __int_as_float(lc[j - 1]));
	cnt[sample] = static_cast<uint8_t>(nc | ((nl - 1) << 4));
}

// Stream-order pass over columns [x0, x1): one thread per row.
__global__ void __launch_bounds__(32) k_bdpt_rows(SceneView sv, const float4 *__restrict__ ref_shade, GiParams p,
                                                  uint32_t *mt_s, int *mt_i, int x0, int x1,
                                                  float4 *__restrict__ rec, uint8_t *__restrict__ cnt, int *status) {
	if (threadIdx.x >= kRowsPerBlock)
		return;
	const int y = blockIdx.x * kRowsPerBlock + threadIdx.x;
	if (y >= p.height)
		return;
	Ctx c{sv, ref_shade, nullptr, 0};
	const GiCam cam = gi_cam(p);
	MtRow rng{mt_s + 624 * static_cast<size_t>(y), mt_i[y]};
	const int cw = x1 - x0;
	for (int x = x0; x < x1; x++) {
		for (int s = 0; s < p.samples; s++) {
			const size_t sample = (static_cast<size_t>(y) * cw + (x - x0)) * p.samples + s;
			record_sample<true>(c, p, cam, x, y, rng, rec, cnt, sample);
		}
	}
	mt_i[y] = rng.i;
	if (c.err)
		atomicOr(status, 1);
}

// Counter streams: every sample is independent, so the subpaths of columns
// [x0, x1) are traced one thread per (pixel, sample) and recorded for the connections.
__global__ void __launch_bounds__(128) k_bdpt_counter_paths(SceneView sv, const float4 *__restrict__ ref_shade,
                                                            GiParams p, int x0, int x1, float4 *__restrict__ rec,
                                                            uint8_t *__restrict__ cnt, int *status) {
	const int cw = x1 - x0;
	const long total = static_cast<long>(cw) * p.height * p.samples;
	const long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (i >= total)
		return;
	const long pix_local = i / p.samples;
	const int s = static_cast<int>(i - pix_local * p.samples);
	const int y = static_cast<int>(pix_local / cw), x = x0 + static_cast<int>(pix_local % cw);
	const long pix = static_cast<long>(y) * p.width + x;
	Ctx c{sv, ref_shade, nullptr, 0};
	CtrDraw d{static_cast<uint32_t>(pix), static_cast<uint32_t>(s), 0u, static_cast<uint32_t>(p.seed),
	          static_cast<uint32_t>(p.seed >> 32), 0, U4{0u, 0u, 0u, 0u}};
	record_sample<false>(c, p, gi_cam(p), x, y, d, rec, cnt, static_cast<size_t>(i));
	if (c.err)
		atomicOr(status, 1);
}

// Rebuilds a recorded subpath: normals and albedos from the triangle codes, the
// throughputs as the same running products the tracing pass formed.
__device__ __forceinline__ V3 replay(const float4 *ref_shade, const float4 *r, int n, V3 beta, GV *out) {
	for (int i = 0; i < n; i++) {
		const float4 v = r[i];
		const int code = __float_as_int(v.w);
		const V3 tn = tri_normal(ref_shade, code >> 1);
		GV g;
		g.p = mk(v.x, v.y, v.z);
		g.n = (code & 1) ? -tn : tn;
		g.albedo = tri_albedo(ref_shade, code >> 1);
		g.beta = beta;
		out[i] = g;
		beta = beta * g.albedo;
	}
	return beta;
}

// ---- connections ----
// Every camera vertex is joined to every light vertex (src/BDPT.cpp:110-134) in
// three passes: k_bdpt_pairs lists the pairs that pass the two cosine tests (each
// sample's in one block, in the reference's (i, j) order), k_bdpt_shadow traces
// one shadow ray per listed pair, k_bdpt_fold sums the contributions per pixel in
// the reference's order from the recorded occlusions. A list entry is
// (sample << 5) | (i * 5 + j).
constexpr int kBdptPairs = kGiMaxDepth * (kGiMaxDepth + 1); // 20 per sample at most

struct ConnView {
	int *pair_base;     // per sample: its first list entry
	uint32_t *pair;     // list entries
	uint8_t *occ;       // per entry: 1 if the shadow ray is blocked
	unsigned *count;    // entries listed
};

__device__ __forceinline__ void replay_sample(const float4 *ref_shade, const float4 *r, int nc, int nls, GV *cv,
                                              GV *lv) {
	const V3 le = mk(30.0f, 30.0f, 30.0f) * gi_light_area();
	replay(ref_shade, r, nc, mk(1.0f, 1.0f, 1.0f), cv);
	const float4 l0 = r[kGiMaxDepth];
	lv[0] = GV{mk(l0.x, l0.y, l0.z), mk(0.0f, -1.0f, 0.0f), mk(0.0f, 0.0f, 0.0f), le};
	replay(ref_shade, r + kGiMaxDepth + 1, nls, le, lv + 1);
}

// The direction, distance and the two cosines of one connection, with the
// reference's operations; false where a cosine test rejects it.
__device__ __forceinline__ bool connection(const GV &cv, const GV &l, V3 &d, float &dist, float &dist2, float &cosC,
                                           float &cosL) {
	d = l.p - cv.p;
	dist2 = dot(d, d);
	dist = sqrtf(dist2);
	d = d / dist;
	cosC = dot(cv.n, d);
	cosL = dot(l.n, -d);
	return !(cosC <= 0.0f || cosL <= 0.0f);
}

__global__ void __launch_bounds__(128) k_bdpt_pairs(const float4 *__restrict__ ref_shade, long samples,
                                                    const float4 *__restrict__ rec, const uint8_t *__restrict__ cnt,
                                                    ConnView cv_) {
	// Every lane of the warp takes part in the prefix sum below (lanes past the last
	// sample list nothing), so no early return.
	const long sample = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
	const bool live = sample < samples;
	uint32_t ok = 0; // bit i * 5 + j
	if (live) {
		const int k = cnt[sample];
		const int nc = k & 15, nls = k >> 4;
		GV cv[kGiMaxDepth], lv[kGiMaxDepth + 1];
		replay_sample(ref_shade, rec + static_cast<size_t>(sample) * kBdptRecordSlots, nc, nls, cv, lv);
		for (int i = 0; i < nc; i++)
			for (int j = 0; j <= nls; j++) {
				V3 d;
				float dist, dist2, cosC, cosL;
				if (connection(cv[i], lv[j], d, dist, dist2, cosC, cosL))
					ok |= 1u << (i * 5 + j);
			}
	}
	// one atomic per warp: the lanes' counts are prefix-summed with shuffles
	const int lane = static_cast<int>(threadIdx.x & 31);
	const int mine = __popc(ok);
	int incl = mine;
	for (int off = 1; off < 32; off <<= 1) {
		const int v = __shfl_up_sync(0xffffffffu, incl, off);
		if (lane >= off)
			incl += v;
	}
	unsigned base = 0;
	if (lane == 31 && incl > 0)
		base = atomicAdd(cv_.count, static_cast<unsigned>(incl));
	base = __shfl_sync(0xffffffffu, base, 31);
	if (!live)
		return;
	const unsigned first = base + static_cast<unsigned>(incl - mine);
	cv_.pair_base[sample] = static_cast<int>(first);
	unsigned e = first;
	for (uint32_t bits = ok; bits; bits &= bits - 1)
		cv_.pair[e++] = (static_cast<uint32_t>(sample) << 5) | static_cast<uint32_t>(__ffs(bits) - 1);
}

__global__ void __launch_bounds__(128) k_bdpt_shadow(SceneView sv, const float4 *__restrict__ ref_shade,
                                                     const float4 *__restrict__ rec, ConnView cv_, int *status) {
	Ctx c{sv, ref_shade, nullptr, 0};
	const unsigned n = *cv_.count;
	for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
		const uint32_t w = cv_.pair[e];
		const size_t sample = w >> 5;
		const int code = static_cast<int>(w & 31u), i = code / 5, j = code % 5;
		const float4 *r = rec + sample * kBdptRecordSlots;
		const float4 a = r[i];
		const int ca = __float_as_int(a.w);
		const V3 tn = tri_normal(ref_shade, ca >> 1);
		GV cvx, lx;
		cvx.p = mk(a.x, a.y, a.z);
		cvx.n = (ca & 1) ? -tn : tn;
		const float4 b = r[kGiMaxDepth + j];
		lx.p = mk(b.x, b.y, b.z);
		if (j == 0) {
			lx.n = mk(0.0f, -1.0f, 0.0f);
		} else {
			const int cb = __float_as_int(b.w);
			const V3 tl = tri_normal(ref_shade, cb >> 1);
			lx.n = (cb & 1) ? -tl : tl;
		}
		V3 d;
		float dist, dist2, cosC, cosL;
		connection(cvx, lx, d, dist, dist2, cosC, cosL);
		cv_.occ[e] = occluded(c, cvx.p + cvx.n * kGiEps, d, dist - 2.0f * kGiEps, -1) ? 1 : 0;
	}
	if (c.err)
		atomicOr(status, 1);
}

// Sums one pixel's connections over its samples in the reference's order: for each
// sample, camera vertex i, light vertex j, contribution x uniform MIS weight.
__global__ void __launch_bounds__(128) k_bdpt_fold(const float4 *__restrict__ ref_shade, GiParams p, int x0, int x1,
                                                   const float4 *__restrict__ rec, const uint8_t *__restrict__ cnt,
                                                   ConnView cv_, uint32_t *argb, float *rgb) {
	const int cw = x1 - x0;
	const long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (idx >= static_cast<long>(cw) * p.height)
		return;
	const int y = static_cast<int>(idx / cw), x = x0 + static_cast<int>(idx % cw);
	V3 acc = mk(0.0f, 0.0f, 0.0f);
	for (int s = 0; s < p.samples; s++) {
		const size_t sample = static_cast<size_t>(idx) * p.samples + s;
		const int k = cnt[sample];
		const int nc = k & 15, nls = k >> 4;
		GV cv[kGiMaxDepth], lv[kGiMaxDepth + 1];
		replay_sample(ref_shade, rec + sample * kBdptRecordSlots, nc, nls, cv, lv);
		unsigned e = static_cast<unsigned>(cv_.pair_base[sample]);
		for (int i = 0; i < nc; i++) {
			const GV c0 = cv[i];
			for (int j = 0; j <= nls; j++) {
				const GV l = lv[j];
				V3 d;
				float dist, dist2, cosC, cosL;
				if (!connection(c0, l, d, dist, dist2, cosC, cosL))
					continue;
				if (cv_.occ[e++])
					continue;
				const float G = cosC * cosL / dist2;
				const V3 fC = c0.albedo / kGiPi;
				V3 contrib = c0.beta * fC * G * l.beta;
				if (j > 0)
					contrib = contrib * (l.albedo / kGiPi);
				const float w = 1.0f / static_cast<float>(i + j + 2);
				acc = acc + contrib * w;
			}
		}
	}
	const V3 col = acc * (p.exposure / static_cast<float>(p.samples));
	gi_store(p, static_cast<long>(y) * p.width + x, col, argb, rgb);
}

// ---- Metropolis ----

__device__ __forceinline__ float luminance(V3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

// The primary-sample vector of one state (src/Metropolis.cpp:26-36): coordinates
// past n are drawn from `ext` on first use.
template <class E> struct MltSampler {
	float *u;
	int &n;
	E &ext;
	int idx;
	__device__ float next() {
		if (idx >= n) {
			u[n] = ext(idx);
			n++;
		}
		return u[idx++];
	}
};

// eval + tracePath with next-event estimation (src/Metropolis.cpp:53-81, 96-105).
template <class S> __device__ V3 mlt_eval(Ctx &c, const GiParams &p, const GiCam &cam, S &smp, int &pixel) {
	const float fx = smp.next(), fy = smp.next();
	const int px = min(p.width - 1, static_cast<int>(fx * static_cast<float>(p.width)));
	const int py = min(p.height - 1, static_cast<int>(fy * static_cast<float>(p.height)));
	pixel = py * p.width + px;
	const float sx = (static_cast<float>(px) + 0.5f - static_cast<float>(p.width) / 2.0f) / p.f;
	const float sy = -(static_cast<float>(py) + 0.5f - static_cast<float>(p.height) / 2.0f) / p.f;
	V3 d = normalize(cam.right * sx + cam.up * sy + cam.fwd * -1.0f);
	V3 o = cam.pos;
	V3 L = mk(0.0f, 0.0f, 0.0f), beta = mk(1.0f, 1.0f, 1.0f);
	const V3 ln = mk(0.0f, -1.0f, 0.0f);
	const V3 le = mk(30.0f, 30.0f, 30.0f);
	for (int depth = 0; depth < kGiMaxDepth; depth++) {
		const Hit h = intersect(c, o, d, -1);
		if (!h.hit)
			break;
		const V3 tn = tri_normal(c.ref_shade, h.idx);
		const V3 n = dot(tn, d) < 0.0f ? tn : -tn;
		const V3 albedo = tri_albedo(c.ref_shade, h.idx);
		const V3 point = h.point;
		// glm::vec3((next * 2 - 1) * half, 0, (next * 2 - 1) * half): right to left
		const float uz = smp.next(), ux = smp.next();
		const V3 lp =
		    mk(0.0f, 0.33f, 0.0f) + mk((ux * 2.0f - 1.0f) * kGiLightHalf, 0.0f, (uz * 2.0f - 1.0f) * kGiLightHalf);
		V3 toL = lp - point;
		const float dist = length(toL);
		toL = toL / dist;
		const float cosS = dot(n, toL), cosL = dot(ln, -toL);
		if (cosS > 0.0f && cosL > 0.0f && !occluded(c, point + n * kGiEps, toL, dist - 2.0f * kGiEps, -1)) {
			const float G = cosS * cosL / (dist * dist);
			L = L + beta * (albedo / kGiPi) * G * le * gi_light_area();
		}
		// cosineHemisphere(n, next, next): right to left, u2 first
		const float u2 = smp.next(), u1 = smp.next();
		const V3 nd = cosine_hemisphere_u(n, u1, u2);
		beta = beta * albedo;
		o = point + kGiEps * nd;
		d = nd;
	}
	return L;
}

// Standard normal from two uniforms (Box and Muller 1958), evaluated in double.
__device__ __forceinline__ float gi_normal(float u1, float u2) {
	return static_cast<float>(sqrt(-2.0 * log(1.0 - static_cast<double>(u1))) *
	                          cos(6.283185307179586 * static_cast<double>(u2)));
}

__global__ void __launch_bounds__(128) k_mlt_bootstrap(SceneView sv, const float4 *__restrict__ ref_shade, GiParams p,
                                                       float *lum, uint8_t *len, int *status) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= p.bootstrap)
		return;
	Ctx c{sv, ref_shade, nullptr, 0};
	const GiCam cam = gi_cam(p);
	CtrDraw d{static_cast<uint32_t>(i), 0u, 1u, static_cast<uint32_t>(p.seed), static_cast<uint32_t>(p.seed >> 32), 0,
	          U4{0u, 0u, 0u, 0u}};
	auto ext = [&](int) { return d(); };
	float u[kMltDims];
	int n = 0, pix = 0;
	MltSampler<decltype(ext)> smp{u, n, ext, 0};
	lum[i] = luminance(mlt_eval(c, p, cam, smp, pix));
	len[i] = static_cast<uint8_t>(n);
	if (c.err)
		atomicOr(status, 1);
}

// Inclusive luminance prefix in double: 1024 contiguous segments, each summed in
// order, then the segment starts in order.
__global__ void __launch_bounds__(1024) k_mlt_cdf(const float *lum, int count, double *cdf, double *total) {
	__shared__ double start[1025];
	const int t = threadIdx.x;
	const int seg = (count + 1023) / 1024;
	const int i0 = t * seg, i1 = min(count, i0 + seg);
	double part = 0.0;
	for (int i = i0; i < i1; i++)
		part += static_cast<double>(lum[i]);
	start[t + 1] = part;
	__syncthreads();
	if (t == 0) {
		double run = 0.0;
		for (int k = 0; k < 1024; k++) {
			const double pk = start[k + 1];
			start[k] = run;
			run += pk;
		}
		start[1024] = run;
		*total = run;
	}
	__syncthreads();
	double run = start[t];
	for (int i = i0; i < i1; i++) {
		run += static_cast<double>(lum[i]);
		cdf[i] = run;
	}
}

// Random words of one chain step: counter (chain, step, k / 4, 3), word k % 4.
struct StepDraw {
	uint32_t chain, step, k0, k1;
	int cached;
	U4 blk;
	__device__ float operator()(int k) {
		if ((k >> 2) != cached) {
			cached = k >> 2;
			blk = philox4x32_10(U4{chain, step, static_cast<uint32_t>(cached), 3u}, k0, k1);
		}
		return canonical01(u4_word(blk, k & 3));
	}
};

__device__ __forceinline__ void deposit(float *image, int pix, V3 v) {
	atomicAdd(image + 3 * static_cast<size_t>(pix), v.x);
	atomicAdd(image + 3 * static_cast<size_t>(pix) + 1, v.y);
	atomicAdd(image + 3 * static_cast<size_t>(pix) + 2, v.z);
}

// One Markov chain per thread (src/Metropolis.cpp:127-173 per chain).
__global__ void __launch_bounds__(128) k_mlt_chains(SceneView sv, const float4 *__restrict__ ref_shade, GiParams p,
                                                    const double *__restrict__ cdf, const double *__restrict__ total,
                                                    const uint8_t *__restrict__ len, float *image, int *status) {
	const int ch = blockIdx.x * blockDim.x + threadIdx.x;
	if (ch >= p.chains)
		return;
	const double tot = *total;
	if (!(tot > 0.0))
		return;
	const uint32_t k0 = static_cast<uint32_t>(p.seed), k1 = static_cast<uint32_t>(p.seed >> 32);
	Ctx c{sv, ref_shade, nullptr, 0};
	const GiCam cam = gi_cam(p);
	// chain start: the bootstrap path whose inclusive prefix first exceeds xi * total
	const float xi = canonical01(philox4x32_10(U4{static_cast<uint32_t>(ch), 0u, 0u, 2u}, k0, k1).x);
	const double target = static_cast<double>(xi) * tot;
	int lo = 0, hi = p.bootstrap - 1;
	while (lo < hi) {
		const int mid = (lo + hi) / 2;
		if (cdf[mid] > target)
			hi = mid;
		else
			lo = mid + 1;
	}
	float cur[kMltDims], prop[kMltDims];
	int cn = len[lo];
	{
		CtrDraw d{static_cast<uint32_t>(lo), 0u, 1u, k0, k1, 0, U4{0u, 0u, 0u, 0u}};
		for (int m = 0; m < cn; m++)
			cur[m] = d();
	}
	int cur_pix = 0;
	auto never = [](int) { return 0.0f; };
	MltSampler<decltype(never)> s0{cur, cn, never, 0};
	V3 curL = mlt_eval(c, p, cam, s0, cur_pix);
	float curLum = luminance(curL);
	const long long steps = p.mutations / p.chains + (ch < p.mutations % p.chains ? 1 : 0);
	const float sigma = 0.02f, p_large = 0.3f;
	for (long long t = 0; t < steps; t++) {
		StepDraw W{static_cast<uint32_t>(ch), static_cast<uint32_t>(t), k0, k1, -1, U4{0u, 0u, 0u, 0u}};
		const bool large = W(0) < p_large;
		int pn = cn;
		for (int m = 0; m < cn; m++) {
			if (large) {
				prop[m] = W(2 + 2 * m);
			} else {
				const float a0 = W(2 + 2 * m), a1 = W(3 + 2 * m);
				float v = cur[m] + sigma * gi_normal(a0, a1);
				v = v - floorf(v);
				prop[m] = v;
			}
		}
		auto ext = [&](int m) { return W(40 + m); };
		MltSampler<decltype(ext)> sp{prop, pn, ext, 0};
		int prop_pix = 0;
		const V3 propL = mlt_eval(c, p, cam, sp, prop_pix);
		const float propLum = luminance(propL);
		float a = 1.0f;
		if (curLum > 0.0f) {
			const float r = propLum / curLum;
			a = (r < 1.0f) ? r : 1.0f; // std::min(1.0f, r)
		}
		if (propLum > 0.0f)
			deposit(image, prop_pix, propL * (a / propLum));
		if (curLum > 0.0f)
			deposit(image, cur_pix, curL * ((1.0f - a) / curLum));
		if (W(1) < a) {
			for (int m = 0; m < pn; m++)
				cur[m] = prop[m];
			cn = pn;
			cur_pix = prop_pix;
			curL = propL;
			curLum = propLum;
		}
	}
	if (c.err)
		atomicOr(status, 1);
}

// Normalisation and the canvas (src/Metropolis.cpp:179-191).
__global__ void k_mlt_resolve(GiParams p, const float *__restrict__ image, const double *__restrict__ total,
                              uint32_t *argb, float *rgb, double *b_out) {
	const double bd = *total / static_cast<double>(p.bootstrap);
	const float b = static_cast<float>(bd);
	const long n = static_cast<long>(p.width) * p.height;
	for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		if (i == 0 && b_out)
			*b_out = bd;
		if (!(b > 0.0f)) {
			argb[i] = 0u; // the cleared canvas the reference leaves
			if (rgb)
				rgb[3 * i] = rgb[3 * i + 1] = rgb[3 * i + 2] = 0.0f;
			continue;
		}
		const float scale =
		    b * static_cast<float>(p.width) * static_cast<float>(p.height) / static_cast<float>(p.mutations);
		const V3 v = mk(image[3 * i], image[3 * i + 1], image[3 * i + 2]) * scale;
		if (rgb) {
			rgb[3 * i] = v.x;
			rgb[3 * i + 1] = v.y;
			rgb[3 * i + 2] = v.z;
		}
		argb[i] = gi_pack(v * p.exposure);
	}
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Bytes per sample of a chunk: its subpath record, its first list entry, and up to
// 20 list entries with their occlusion bytes.
constexpr size_t kBdptSampleBytes = kBdptRecordBytes + 4 + kBdptPairs * 5;

int bdpt_chunk_width(const GiParams &p, size_t budget) {
	const size_t per_col = static_cast<size_t>(p.height) * static_cast<size_t>(p.samples);
	size_t cw = per_col ? budget / (per_col * kBdptSampleBytes) : 1;
	// list entries hold the sample index in 27 bits
	if (per_col)
		cw = std::min(cw, (size_t(1) << 27) / per_col);
	cw = std::max<size_t>(1, std::min<size_t>(cw, static_cast<size_t>(p.width)));
	return static_cast<int>(cw);
}

} // namespace

size_t bdpt_scratch_bytes(const GiParams &p, bool reference_stream, size_t chunk_budget) {
	(void)reference_stream; // both streams record subpaths; the row streams' state is small
	const size_t rows = static_cast<size_t>(p.height);
	const size_t samples = static_cast<size_t>(bdpt_chunk_width(p, chunk_budget)) * rows * p.samples;
	return align256(624 * 4 * rows) + align256(4 * rows) + align256(samples * kBdptRecordSlots * 16) +
	       align256(samples) + align256(samples * 4) + align256(samples * kBdptPairs * 4) +
	       align256(samples * kBdptPairs) + 256;
}

cudaError_t launch_bdpt(const SceneView &sv, const float4 *ref_shade, const GiParams &p, bool reference_stream,
                        size_t chunk_budget, void *scratch, uint32_t *argb, float *rgb, int *status, cudaStream_t st) {
	const size_t rows = static_cast<size_t>(p.height);
	const int cw = bdpt_chunk_width(p, chunk_budget);
	const size_t samples = static_cast<size_t>(cw) * rows * p.samples;
	char *base = static_cast<char *>(scratch);
	uint32_t *mt_s = reinterpret_cast<uint32_t *>(base);
	base += align256(624 * 4 * rows);
	int *mt_i = reinterpret_cast<int *>(base);
	base += align256(4 * rows);
	float4 *rec = reinterpret_cast<float4 *>(base);
	base += align256(samples * kBdptRecordSlots * 16);
	uint8_t *cnt = reinterpret_cast<uint8_t *>(base);
	base += align256(samples);
	ConnView cv;
	cv.pair_base = reinterpret_cast<int *>(base);
	base += align256(samples * 4);
	cv.pair = reinterpret_cast<uint32_t *>(base);
	base += align256(samples * kBdptPairs * 4);
	cv.occ = reinterpret_cast<uint8_t *>(base);
	base += align256(samples * kBdptPairs);
	cv.count = reinterpret_cast<unsigned *>(base);
	if (reference_stream)
		k_mt_seed_rows<<<static_cast<unsigned>((rows + 127) / 128), 128, 0, st>>>(mt_s, mt_i, p.height);
	for (int x0 = 0; x0 < p.width; x0 += cw) {
		const int x1 = std::min(p.width, x0 + cw);
		if (reference_stream) {
			TraceRange r("subpaths in row-stream order");
			k_bdpt_rows<<<static_cast<unsigned>((rows + kRowsPerBlock - 1) / kRowsPerBlock), 32, 0, st>>>(
			    sv, ref_shade, p, mt_s, mt_i, x0, x1, rec, cnt, status);
		} else {
			TraceRange r("subpaths, one thread per sample");
			const long n = static_cast<long>(x1 - x0) * p.height * p.samples;
			k_bdpt_counter_paths<<<static_cast<unsigned>((n + 127) / 128), 128, 0, st>>>(sv, ref_shade, p, x0, x1,
			                                                                            rec, cnt, status);
		}
		TraceRange r("connections");
		const long ns = static_cast<long>(x1 - x0) * p.height * p.samples;
		const long npx = static_cast<long>(x1 - x0) * p.height;
		cudaError_t e = cudaMemsetAsync(cv.count, 0, sizeof(unsigned), st);
		if (e != cudaSuccess)
			return e;
		k_bdpt_pairs<<<static_cast<unsigned>((ns + 127) / 128), 128, 0, st>>>(ref_shade, ns, rec, cnt, cv);
		k_bdpt_shadow<<<148 * 16, 128, 0, st>>>(sv, ref_shade, rec, cv, status);
		k_bdpt_fold<<<static_cast<unsigned>((npx + 127) / 128), 128, 0, st>>>(ref_shade, p, x0, x1, rec, cnt, cv, argb,
		                                                                      rgb);
	}
	return cudaGetLastError();
}

size_t mlt_scratch_bytes(const GiParams &p) {
	const size_t b = static_cast<size_t>(p.bootstrap);
	return align256(b * 4) + align256(b) + align256(b * 8) + 256 +
	       align256(static_cast<size_t>(p.width) * p.height * 3 * 4);
}

cudaError_t launch_mlt(const SceneView &sv, const float4 *ref_shade, const GiParams &p, void *scratch, uint32_t *argb,
                       float *rgb, double *b_out, int *status, cudaStream_t st) {
	const size_t b = static_cast<size_t>(p.bootstrap);
	const long npix = static_cast<long>(p.width) * p.height;
	char *base = static_cast<char *>(scratch);
	float *lum = reinterpret_cast<float *>(base);
	base += align256(b * 4);
	uint8_t *len = reinterpret_cast<uint8_t *>(base);
	base += align256(b);
	double *cdf = reinterpret_cast<double *>(base);
	base += align256(b * 8);
	double *total = reinterpret_cast<double *>(base);
	base += 256;
	float *image = reinterpret_cast<float *>(base);
	cudaError_t e = cudaMemsetAsync(image, 0, static_cast<size_t>(npix) * 3 * 4, st);
	if (e != cudaSuccess)
		return e;
	{
		TraceRange r("bootstrap");
		k_mlt_bootstrap<<<static_cast<unsigned>((b + 127) / 128), 128, 0, st>>>(sv, ref_shade, p, lum, len, status);
		k_mlt_cdf<<<1, 1024, 0, st>>>(lum, p.bootstrap, cdf, total);
	}
	TraceRange r("chains");
	k_mlt_chains<<<static_cast<unsigned>((p.chains + 127) / 128), 128, 0, st>>>(sv, ref_shade, p, cdf, total, len,
	                                                                          image, status);
	const long g = std::min<long>((npix + 255) / 256, 148 * 16);
	k_mlt_resolve<<<static_cast<unsigned>(g), 256, 0, st>>>(p, image, total, argb, rgb, b_out);
	return cudaGetLastError();
}

} // namespace rnb
