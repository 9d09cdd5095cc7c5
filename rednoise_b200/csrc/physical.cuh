// Physical-mode path tracing: the per-vertex logic shared by the megakernel,
// the wavefront stages and the adjoint replay.
//
// Estimator (the additive API's semantics; the CPU oracle restates it):
//   * camera: pinhole, vertical FOV, jitter (u0, u1) of counter block 0;
//   * vertex b (hit by the ray of depth b): emission of a front-facing emitter
//     triangle with MIS (power heuristic) against light sampling, emitters absorb;
//     next-event estimation to one emitter triangle chosen by area, point uniform
//     on it, shadow ray, MIS weight; BSDF sampling: Lambert (cosine), GGX metal
//     (visible-normal sampling, Heitz 2018; height-correlated Smith G2; Schlick
//     Fresnel with F0 = albedo), smooth dielectric (exact Fresnel, reflect or
//     refract by its probability); Russian roulette from depth rr_depth with
//     survival min(0.95, max(throughput));
//   * uniforms of vertex b: blocks 2 + 2b (light select, light u, light v, lobe)
//     and 3 + 2b (direction u, direction v, roulette, -).
// Triangles whose emission is positive are lights: they are hit but absorb.
//
// Arithmetic contract: the translation units that include this file are compiled
// without multiply-add contraction (-fmad=false), divisions and square roots are
// IEEE, and sin/cos are sincos_turn's plain float operations, so every path's
// radiance is the bit pattern the CPU restatement (compiled without contraction)
// computes for the same uniforms.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rng.cuh"
#include "traverse.cuh"

namespace rnb {

struct PhysScene {
	SceneView sv;
	const float4 *__restrict__ shade;    // 3 per triangle: (albedo, material), (Le, param), (normal, emitter flag)
	const float4 *__restrict__ emitters; // 3 per emitter: (v0, tri), (e0, area), (e1, cdf)
	int n_emitters;
	float emit_area_total;
};

struct PhysCamera {
	float pos[3];
	float fwd[3], right[3], up[3];
	float tan_half_y; // tan(vfov / 2)
	float aspect;     // width / height
	int width, height;
};

struct PhysSettings {
	int spp;
	int max_depth; // scattering vertices per path
	int rr_depth;  // first vertex index with Russian roulette
	int order;     // TraversalOrder for closest hits
	unsigned long long seed;
	uint32_t sample_offset;
	float env[3];
};

#ifdef __CUDACC__

struct F3 {
	float x, y, z;
};
__device__ __forceinline__ F3 f3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 operator-(F3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ F3 operator*(F3 a, F3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ F3 operator*(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ F3 operator*(float s, F3 a) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
	return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// 1 / sqrt with IEEE division and square root (not the approximate rsqrtf), so a
// unit vector carries the same bits as the CPU restatement's a * (1 / std::sqrt(a.a)).
__device__ __forceinline__ F3 norm3(F3 a) { return a * (1.0f / sqrtf(dot3(a, a))); }
__device__ __forceinline__ float maxc(F3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
__device__ __forceinline__ F3 ld3(const float4 v) { return {v.x, v.y, v.z}; }

// sin(2 pi u) and cos(2 pi u) for u in [0, 1): the angle is reduced exactly to a
// quarter turn q and a remainder f in [-1/2, 1/2] quarter turns (scaling by 4 and
// removing the integer part are exact in float), x = f pi / 2 with |x| <= pi / 4,
// then the Taylor series of sin to x^11 and of cos to x^12 (the omitted terms are
// below 7e-12 there) and the quadrant's rotation. Written with plain IEEE float
// operations only, so a CPU compiled without contraction computes the same bits;
// about one ulp from the exact values.
__device__ __forceinline__ void sincos_turn(float u, float &s, float &c) {
	const float t = u * 4.0f;
	int q = static_cast<int>(t);
	float f = t - static_cast<float>(q);
	if (f > 0.5f) {
		f = f - 1.0f;
		q = q + 1;
	}
	const float x = f * 1.57079632679489662f;
	const float x2 = x * x;
	const float sp =
	    x + x * x2 *
	            (-1.66666666666666667e-1f +
	             x2 * (8.33333333333333333e-3f +
	                   x2 * (-1.98412698412698413e-4f + x2 * (2.75573192239858907e-6f + x2 * -2.50521083854417188e-8f))));
	const float cp =
	    1.0f + x2 * (-0.5f + x2 * (4.16666666666666667e-2f +
	                               x2 * (-1.38888888888888889e-3f +
	                                     x2 * (2.48015873015873016e-5f +
	                                           x2 * (-2.75573192239858907e-7f + x2 * 2.08767569878680990e-9f)))));
	switch (q & 3) {
	case 0:
		s = sp;
		c = cp;
		break;
	case 1:
		s = cp;
		c = -sp;
		break;
	case 2:
		s = -sp;
		c = -cp;
		break;
	default:
		s = -cp;
		c = sp;
		break;
	}
}

// Orthonormal basis around n (Duff et al., "Building an Orthonormal Basis, Revisited", 2017).
__device__ __forceinline__ void onb(F3 n, F3 &t, F3 &b) {
	const float sign = copysignf(1.0f, n.z);
	const float a = -1.0f / (sign + n.z);
	const float bb = n.x * n.y * a;
	t = f3(1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x);
	b = f3(bb, sign + n.y * n.y * a, -n.y);
}

struct PathState {
	F3 o, d;
	F3 beta;
	F3 L;
	float prev_pdf; // solid-angle pdf of the BSDF sample that produced the ray; 0 = camera or specular
	int ignore;
	int bounce;
	uint32_t pixel, sample;
};

struct ShadowReq {
	F3 o, d;
	float tmax;
	F3 contrib;
	int ignore;
	bool valid;
};

__device__ __forceinline__ PathState camera_path(const PhysCamera &c, const PhysSettings &s, uint32_t pixel,
                                                 uint32_t sample) {
	const U4 r = path_rand(s.seed, pixel, sample, 0u);
	const int px = static_cast<int>(pixel % static_cast<uint32_t>(c.width));
	const int py = static_cast<int>(pixel / static_cast<uint32_t>(c.width));
	const float sx = ((static_cast<float>(px) + u01(r.x)) / static_cast<float>(c.width)) * 2.0f - 1.0f;
	const float sy = 1.0f - ((static_cast<float>(py) + u01(r.y)) / static_cast<float>(c.height)) * 2.0f;
	const F3 fwd = f3(c.fwd[0], c.fwd[1], c.fwd[2]);
	const F3 right = f3(c.right[0], c.right[1], c.right[2]);
	const F3 up = f3(c.up[0], c.up[1], c.up[2]);
	PathState p;
	p.o = f3(c.pos[0], c.pos[1], c.pos[2]);
	p.d = norm3(fwd + right * (sx * c.tan_half_y * c.aspect) + up * (sy * c.tan_half_y));
	p.beta = f3(1.0f, 1.0f, 1.0f);
	p.L = f3(0.0f, 0.0f, 0.0f);
	p.prev_pdf = 0.0f;
	p.ignore = -1;
	p.bounce = 0;
	p.pixel = pixel;
	p.sample = sample;
	return p;
}

// GGX with height-correlated Smith masking.
__device__ __forceinline__ float ggx_D(float cos_m, float a2) {
	const float k = cos_m * cos_m * (a2 - 1.0f) + 1.0f;
	return a2 / (3.14159265358979f * k * k);
}
__device__ __forceinline__ float ggx_lambda(float cos_w, float a2) {
	const float c2 = cos_w * cos_w;
	const float t2 = fmaxf(0.0f, 1.0f - c2) / fmaxf(c2, 1e-12f);
	return 0.5f * (-1.0f + sqrtf(1.0f + a2 * t2));
}
__device__ __forceinline__ F3 schlick(F3 f0, float c) {
	const float m = fminf(fmaxf(1.0f - c, 0.0f), 1.0f);
	const float m5 = (m * m) * (m * m) * m;
	return f0 + (f3(1.0f, 1.0f, 1.0f) - f0) * m5;
}

// Schlick's (1 - cos)^5 term.
__device__ __forceinline__ float schlick_m5(float c) {
	const float m = fminf(fmaxf(1.0f - c, 0.0f), 1.0f);
	return (m * m) * (m * m) * m;
}

// d log(weight) / d albedo, per channel, of a vertex whose weight is linear in
// the albedo (Lambert) or the Schlick Fresnel of F0 = albedo (GGX, m5 given).
__device__ __forceinline__ F3 albedo_log_derivative(int mat, F3 albedo, float m5) {
	if (mat == 0)
		return f3(1.0f / fmaxf(albedo.x, 1e-12f), 1.0f / fmaxf(albedo.y, 1e-12f), 1.0f / fmaxf(albedo.z, 1e-12f));
	if (mat == 1) {
		const F3 F = albedo + (f3(1.0f, 1.0f, 1.0f) - albedo) * m5;
		const float d = 1.0f - m5;
		return f3(d / fmaxf(F.x, 1e-12f), d / fmaxf(F.y, 1e-12f), d / fmaxf(F.z, 1e-12f));
	}
	return f3(0.0f, 0.0f, 0.0f);
}

// BSDF value times |cos wi| and solid-angle pdf for a non-delta material in the
// local frame of n (wo, wi on the same side as n). Returns false if zero.
// m5 receives Schlick's (1 - wo.m)^5 of the GGX half vector (0 for Lambert).
__device__ __forceinline__ bool bsdf_eval(int mat, F3 albedo, float alpha, F3 n, F3 wo, F3 wi, F3 &f_cos,
                                          float &pdf, float &m5) {
	const float ci = dot3(n, wi), co = dot3(n, wo);
	m5 = 0.0f;
	if (ci <= 0.0f || co <= 0.0f)
		return false;
	if (mat == 0) {
		f_cos = albedo * (ci * 0.318309886183791f);
		pdf = ci * 0.318309886183791f;
		return true;
	}
	const float a2 = alpha * alpha;
	const F3 m = norm3(wo + wi);
	const float cm = dot3(n, m), om = dot3(wo, m);
	if (cm <= 0.0f || om <= 0.0f)
		return false;
	const float D = ggx_D(cm, a2);
	const float lo = ggx_lambda(co, a2), li = ggx_lambda(ci, a2);
	const float G2 = 1.0f / (1.0f + lo + li);
	const float G1 = 1.0f / (1.0f + lo);
	m5 = schlick_m5(om);
	f_cos = schlick(albedo, om) * (D * G2 / (4.0f * co));
	pdf = G1 * D / (4.0f * co);
	return true;
}

// What the adjoint replay needs from one vertex (path replay backpropagation):
// the terms this vertex adds and the log-derivatives of its weights.
struct VertexGrad {
	int tri;          // scattering triangle, -1 if none
	int hit_emitter;  // emitter triangle hit by the incoming ray, -1 if none
	F3 emit;          // emission added at this vertex
	F3 Le;            // radiance of the hit emitter
	bool nee;         // a shadow request was made
	F3 nee_contrib;   // its contribution (added when unoccluded)
	F3 nee_dlog;      // d log f(light direction) / d albedo
	int nee_emitter;  // sampled emitter triangle
	F3 nee_Le;        // its radiance
	F3 cont_dlog;     // d log(continuation weight) / d albedo
};

// Adjoint helpers shared by the per-path and the wavefront adjoint: a / b per channel
// where b > 0 (else 0), and a gradient 3-vector added to one triangle's three floats
// (zero components skipped).
__device__ __forceinline__ F3 safe_div(F3 a, F3 b) {
	return f3(b.x > 0.0f ? a.x / b.x : 0.0f, b.y > 0.0f ? a.y / b.y : 0.0f, b.z > 0.0f ? a.z / b.z : 0.0f);
}
__device__ __forceinline__ void add_grad3(float *p, F3 v) {
	if (v.x != 0.0f)
		atomicAdd(p, v.x);
	if (v.y != 0.0f)
		atomicAdd(p + 1, v.y);
	if (v.z != 0.0f)
		atomicAdd(p + 2, v.z);
}

__device__ __forceinline__ float power_mis(float a, float b) {
	const float a2 = a * a, b2 = b * b;
	return a2 / (a2 + b2);
}

// Shade the vertex the path's ray hit (h), add emission, build the NEE shadow
// request, sample the continuation. Returns whether the path continues. With
// kGrad the terms the adjoint replay needs are recorded in *vg; the decisions
// and arithmetic of the primal are the same either way.
template <bool kGrad>
__device__ __forceinline__ bool shade_vertex_t(const PhysScene &sc, const PhysSettings &st, PathState &ps,
                                               const HitRec &h, ShadowReq &sr, VertexGrad *vg) {
	sr.valid = false;
	if (kGrad) {
		vg->tri = -1;
		vg->hit_emitter = -1;
		vg->nee = false;
		vg->nee_emitter = -1;
		vg->cont_dlog = f3(0.0f, 0.0f, 0.0f);
	}
	if (h.idx < 0) {
		ps.L = ps.L + ps.beta * f3(st.env[0], st.env[1], st.env[2]);
		return false;
	}
	const float4 s0 = __ldg(sc.shade + 3 * static_cast<size_t>(h.idx));
	const float4 s1 = __ldg(sc.shade + 3 * static_cast<size_t>(h.idx) + 1);
	const float4 s2 = __ldg(sc.shade + 3 * static_cast<size_t>(h.idx) + 2);
	const F3 ng = ld3(s2);
	const F3 p = ps.o + ps.d * h.t;
	const F3 wo = -ps.d;
	const float cos_o_g = dot3(ng, wo);
	const F3 Le = ld3(s1);
	if (s2.w != 0.0f) { // emitter flag, fixed when the scene was prepared
		if (cos_o_g > 0.0f) {
			float w = 1.0f;
			if (ps.prev_pdf > 0.0f) {
				const float pdf_light = h.t * h.t / (cos_o_g * sc.emit_area_total);
				w = power_mis(ps.prev_pdf, pdf_light);
			}
			const F3 e = ps.beta * Le * w;
			ps.L = ps.L + e;
			if (kGrad) {
				vg->hit_emitter = h.idx;
				vg->emit = e;
				vg->Le = Le;
			}
		}
		return false;
	}
	if (kGrad)
		vg->tri = h.idx;
	const int mat = __float_as_int(s0.w);
	const F3 albedo = ld3(s0);
	const float param = s1.w;
	const F3 n = cos_o_g >= 0.0f ? ng : -ng; // faces the incoming side
	const uint32_t b = static_cast<uint32_t>(ps.bounce);
	const U4 rA = path_rand(st.seed, ps.pixel, ps.sample, 2u + 2u * b);
	const U4 rB = path_rand(st.seed, ps.pixel, ps.sample, 3u + 2u * b);
	const float eps = 2e-4f;

	// Next-event estimation (non-delta materials).
	if (mat != 2 && sc.n_emitters > 0) {
		const float target = u01(rA.x) * sc.emit_area_total;
		int lo = 0, hi = sc.n_emitters - 1;
		while (lo < hi) { // first emitter whose cumulative area exceeds target
			const int mid = (lo + hi) >> 1;
			if (__ldg(sc.emitters + 3 * mid + 2).w > target)
				hi = mid;
			else
				lo = mid + 1;
		}
		const float4 E0 = __ldg(sc.emitters + 3 * lo);
		const float4 E1 = __ldg(sc.emitters + 3 * lo + 1);
		const float4 E2 = __ldg(sc.emitters + 3 * lo + 2);
		const float su = sqrtf(u01(rA.y));
		const float b1 = u01(rA.z) * su, b2 = 1.0f - su;
		const F3 e0 = ld3(E1), e1 = ld3(E2);
		const F3 q = ld3(E0) + e0 * b1 + e1 * b2;
		F3 wi = q - p;
		const float dist2 = dot3(wi, wi);
		const float dist = sqrtf(dist2);
		wi = wi * (1.0f / dist);
		const int etri = __float_as_int(E0.w);
		const F3 ne = ld3(__ldg(sc.shade + 3 * static_cast<size_t>(etri) + 2));
		const float cos_l = -dot3(ne, wi);
		F3 f_cos;
		float pdf_b, m5;
		if (cos_l > 0.0f && dist > 0.0f && bsdf_eval(mat, albedo, param, n, wo, wi, f_cos, pdf_b, m5)) {
			const float pdf_l = dist2 / (cos_l * sc.emit_area_total);
			const F3 eLe = ld3(__ldg(sc.shade + 3 * static_cast<size_t>(etri) + 1));
			const float w = power_mis(pdf_l, pdf_b);
			sr.o = p + n * eps;
			sr.d = wi;
			sr.tmax = dist;
			sr.ignore = etri;
			sr.contrib = ps.beta * f_cos * eLe * (w / pdf_l);
			sr.valid = true;
			if (kGrad) {
				vg->nee = true;
				vg->nee_contrib = sr.contrib;
				vg->nee_dlog = albedo_log_derivative(mat, albedo, m5);
				vg->nee_emitter = etri;
				vg->nee_Le = eLe;
			}
		}
	}
	if (ps.bounce + 1 >= st.max_depth)
		return false;

	// Sample the continuation.
	F3 wi;
	F3 weight;
	float pdf = 0.0f;
	if (mat == 0) {
		const float r = sqrtf(u01(rB.x));
		float sn, cs;
		sincos_turn(u01(rB.y), sn, cs);
		F3 t, bt;
		onb(n, t, bt);
		const float z = sqrtf(fmaxf(0.0f, 1.0f - u01(rB.x)));
		wi = t * (r * cs) + bt * (r * sn) + n * z;
		const float ci = dot3(wi, n);
		if (ci <= 0.0f)
			return false;
		weight = albedo;
		pdf = ci * 0.318309886183791f;
		if (kGrad)
			vg->cont_dlog = albedo_log_derivative(0, albedo, 0.0f);
	} else if (mat == 1) {
		const float alpha = param, a2 = alpha * alpha;
		F3 t, bt;
		onb(n, t, bt);
		const F3 wl = f3(dot3(wo, t), dot3(wo, bt), dot3(wo, n)); // local wo
		// Visible-normal sampling (Heitz 2018).
		const F3 vh = norm3(f3(alpha * wl.x, alpha * wl.y, wl.z));
		const float lensq = vh.x * vh.x + vh.y * vh.y;
		const F3 T1 = lensq > 0.0f ? f3(-vh.y, vh.x, 0.0f) * (1.0f / sqrtf(lensq)) : f3(1.0f, 0.0f, 0.0f);
		const F3 T2 = cross3(vh, T1);
		const float r = sqrtf(u01(rB.x));
		float sn, cs;
		sincos_turn(u01(rB.y), sn, cs);
		const float t1 = r * cs;
		float t2 = r * sn;
		const float sblend = 0.5f * (1.0f + vh.z);
		t2 = (1.0f - sblend) * sqrtf(fmaxf(0.0f, 1.0f - t1 * t1)) + sblend * t2;
		const F3 nh = T1 * t1 + T2 * t2 + vh * sqrtf(fmaxf(0.0f, 1.0f - t1 * t1 - t2 * t2));
		const F3 ml = norm3(f3(alpha * nh.x, alpha * nh.y, fmaxf(0.0f, nh.z)));
		const F3 m = t * ml.x + bt * ml.y + n * ml.z;
		const float om = dot3(wo, m);
		wi = m * (2.0f * om) - wo;
		const float ci = dot3(wi, n), co = wl.z;
		if (ci <= 0.0f || om <= 0.0f || co <= 0.0f)
			return false;
		const float lo_ = ggx_lambda(co, a2), li_ = ggx_lambda(ci, a2);
		const float G1 = 1.0f / (1.0f + lo_);
		const float G2 = 1.0f / (1.0f + lo_ + li_);
		weight = schlick(albedo, om) * (G2 / G1);
		pdf = G1 * ggx_D(ml.z, a2) / (4.0f * co);
		if (kGrad)
			vg->cont_dlog = albedo_log_derivative(1, albedo, schlick_m5(om));
	} else {
		// Smooth dielectric: exact Fresnel, choose reflection with probability F.
		const float eta = param;
		const bool entering = cos_o_g > 0.0f;
		const float eta_i = entering ? 1.0f : eta, eta_t = entering ? eta : 1.0f;
		const float ci = fabsf(cos_o_g);
		const float rel = eta_i / eta_t;
		const float s2t = rel * rel * fmaxf(0.0f, 1.0f - ci * ci);
		float F = 1.0f, ct = 0.0f;
		if (s2t < 1.0f) {
			ct = sqrtf(1.0f - s2t);
			const float rs = (eta_i * ci - eta_t * ct) / (eta_i * ci + eta_t * ct);
			const float rp = (eta_t * ci - eta_i * ct) / (eta_t * ci + eta_i * ct);
			F = 0.5f * (rs * rs + rp * rp);
		}
		if (u01(rA.w) < F) {
			wi = n * (2.0f * ci) - wo;
		} else {
			wi = ps.d * rel + n * (rel * ci - ct);
		}
		weight = f3(1.0f, 1.0f, 1.0f);
		pdf = 0.0f;
	}
	ps.beta = ps.beta * weight;
	if (ps.bounce + 1 >= st.rr_depth) {
		const float q = fminf(0.95f, maxc(ps.beta));
		if (!(u01(rB.z) < q))
			return false;
		ps.beta = ps.beta * (1.0f / q);
	}
	const float side = dot3(wi, ng) >= 0.0f ? 1.0f : -1.0f;
	ps.o = p + ng * (side * eps);
	ps.d = wi;
	ps.prev_pdf = pdf;
	ps.ignore = h.idx;
	ps.bounce++;
	return true;
}

__device__ __forceinline__ bool shade_vertex(const PhysScene &sc, const PhysSettings &st, PathState &ps,
                                             const HitRec &h, ShadowReq &sr) {
	return shade_vertex_t<false>(sc, st, ps, h, sr, nullptr);
}

#endif // __CUDACC__

} // namespace rnb
