// Path-replay adjoint of the physical estimator (path replay backpropagation,
// Vicini, Speierer, Jakob 2021): d(loss)/d(per-triangle albedo) and
// d(loss)/d(per-triangle emitted radiance) with O(1) memory per path.
//
// A path is identified by its counter-based RNG key (pixel, sample), so the
// adjoint regenerates it instead of storing vertices. Each sample is traced
// twice: pass 1 computes the path's radiance C; pass 2 replays the same
// decisions and, at every vertex k with albedo a_k, adds
//     g * (N_k * dlog f_k(light)/da_k + (C - P_k) * dlog w_k/da_k)
// to dL/da[tri_k], where g = dL/dI(pixel) / spp, N_k is the vertex's next-event
// term, P_k the radiance gathered up to and including vertex k, and w_k the
// continuation weight (albedo for Lambert, F G2/G1 for GGX). Emission terms E add
// g * E / Le to dL/dLe of their emitter. Roulette probabilities are treated as
// constants. Small scenes accumulate in shared memory and flush once per block;
// large scenes add straight to global memory (red.global.add.f32).
#include "adjoint.hpp"

namespace rnb {

namespace {

__device__ __forceinline__ int find_view(const AdjView *v, int n, int gp) {
	int lo = 0, hi = n - 1;
	while (lo < hi) {
		const int mid = (lo + hi + 1) >> 1;
		if (v[mid].pix_base <= gp)
			lo = mid;
		else
			hi = mid - 1;
	}
	return lo;
}

template <bool kShared>
__device__ __forceinline__ void add3(float *gbuf, float *sbuf, int tri, F3 v) {
	float *p = kShared ? sbuf + 3 * tri : gbuf + 3 * static_cast<size_t>(tri);
	if (v.x != 0.0f)
		atomicAdd(p, v.x);
	if (v.y != 0.0f)
		atomicAdd(p + 1, v.y);
	if (v.z != 0.0f)
		atomicAdd(p + 2, v.z);
}

__device__ __forceinline__ F3 safe_div(F3 a, F3 b) {
	return f3(b.x > 0.0f ? a.x / b.x : 0.0f, b.y > 0.0f ? a.y / b.y : 0.0f, b.z > 0.0f ? a.z / b.z : 0.0f);
}

template <bool kShared>
__global__ void __launch_bounds__(128) k_adjoint(PhysScene sc, const AdjView *__restrict__ views, int n_views,
                                                 int total_pix, float *__restrict__ d_alb, float *__restrict__ d_em,
                                                 int n_tris, int *status) {
	extern __shared__ float smem[];
	float *s_alb = smem;
	float *s_em = smem + 3 * n_tris;
	if (kShared) {
		for (int i = threadIdx.x; i < 6 * n_tris; i += blockDim.x)
			smem[i] = 0.0f;
		__syncthreads();
	}
	int err = 0;
	for (int gp = blockIdx.x * blockDim.x + threadIdx.x; gp < total_pix; gp += gridDim.x * blockDim.x) {
		const int vi = find_view(views, n_views, gp);
		const AdjView &view = views[vi];
		const int pix = gp - view.pix_base;
		const float inv = view.st.spp > 0 ? 1.0f / static_cast<float>(view.st.spp) : 0.0f;
		const F3 g = f3(view.dimg[3 * pix] * inv, view.dimg[3 * pix + 1] * inv, view.dimg[3 * pix + 2] * inv);
		if (g.x == 0.0f && g.y == 0.0f && g.z == 0.0f)
			continue;
		for (int s = 0; s < view.st.spp; s++) {
			const uint32_t sample = view.st.sample_offset + static_cast<uint32_t>(s);
			// Pass 1: the path's radiance.
			PathState ps = camera_path(view.cam, view.st, static_cast<uint32_t>(pix), sample);
			for (;;) {
				const RayPre r = make_ray(ps.o.x, ps.o.y, ps.o.z, ps.d.x, ps.d.y, ps.d.z);
				const HitRec h = trace_closest_best<kOrderReference>(sc.sv, r, ps.ignore, err);
				ShadowReq sr;
				const bool alive = shade_vertex(sc, view.st, ps, h, sr);
				if (sr.valid) {
					const RayPre rs = make_ray(sr.o.x, sr.o.y, sr.o.z, sr.d.x, sr.d.y, sr.d.z);
					if (!trace_any_best(sc.sv, rs, sr.tmax, sr.ignore, err))
						ps.L = ps.L + sr.contrib;
				}
				if (!alive)
					break;
			}
			const F3 C = ps.L;
			if (C.x == 0.0f && C.y == 0.0f && C.z == 0.0f)
				continue; // a path that carries no radiance has no derivative
			// Pass 2: replay and scatter the derivatives.
			ps = camera_path(view.cam, view.st, static_cast<uint32_t>(pix), sample);
			F3 P = f3(0.0f, 0.0f, 0.0f);
			for (;;) {
				const RayPre r = make_ray(ps.o.x, ps.o.y, ps.o.z, ps.d.x, ps.d.y, ps.d.z);
				const HitRec h = trace_closest_best<kOrderReference>(sc.sv, r, ps.ignore, err);
				ShadowReq sr;
				VertexGrad vg;
				const bool alive = shade_vertex_t<true>(sc, view.st, ps, h, sr, &vg);
				if (vg.hit_emitter >= 0) {
					P = P + vg.emit;
					add3<kShared>(d_em, s_em, vg.hit_emitter, g * safe_div(vg.emit, vg.Le));
				}
				if (sr.valid) {
					const RayPre rs = make_ray(sr.o.x, sr.o.y, sr.o.z, sr.d.x, sr.d.y, sr.d.z);
					if (!trace_any_best(sc.sv, rs, sr.tmax, sr.ignore, err)) {
						P = P + vg.nee_contrib;
						add3<kShared>(d_alb, s_alb, vg.tri, g * vg.nee_contrib * vg.nee_dlog);
						add3<kShared>(d_em, s_em, vg.nee_emitter, g * safe_div(vg.nee_contrib, vg.nee_Le));
					}
				}
				if (!alive)
					break;
				add3<kShared>(d_alb, s_alb, vg.tri, g * (C - P) * vg.cont_dlog);
			}
		}
	}
	if (kShared) {
		__syncthreads();
		for (int i = threadIdx.x; i < 3 * n_tris; i += blockDim.x) {
			if (s_alb[i] != 0.0f)
				atomicAdd(d_alb + i, s_alb[i]);
			if (s_em[i] != 0.0f)
				atomicAdd(d_em + i, s_em[i]);
		}
	}
	if (err)
		atomicOr(status, 1);
}

} // namespace

cudaError_t launch_adjoint(const PhysScene &sc, const AdjView *d_views, int n_views, int total_pix, float *d_alb,
                           float *d_em, int n_tris, int *status, cudaStream_t st) {
	if (total_pix <= 0)
		return cudaSuccess;
	int dev = 0, sms = 148;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	const size_t smem = static_cast<size_t>(6) * n_tris * sizeof(float);
	const bool shared = n_tris <= kAdjointSharedTris;
	int per_sm = 0;
	if (shared) {
		cudaFuncSetAttribute(k_adjoint<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adjoint<true>, 128, smem);
	} else {
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adjoint<false>, 128, 0);
	}
	if (per_sm < 1)
		per_sm = 1;
	int blocks = sms * per_sm;
	const int need = (total_pix + 127) / 128;
	if (blocks > need)
		blocks = need;
	if (shared)
		k_adjoint<true><<<blocks, 128, smem, st>>>(sc, d_views, n_views, total_pix, d_alb, d_em, n_tris, status);
	else
		k_adjoint<false><<<blocks, 128, 0, st>>>(sc, d_views, n_views, total_pix, d_alb, d_em, n_tris, status);
	return cudaGetLastError();
}

__global__ void k_set_materials(float4 *shade, int n, const float *__restrict__ albedo,
                                const float *__restrict__ emission) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		if (albedo) {
			float4 a = shade[3 * i];
			a.x = albedo[3 * i];
			a.y = albedo[3 * i + 1];
			a.z = albedo[3 * i + 2];
			shade[3 * i] = a;
		}
		if (emission) {
			// Emitter membership (the flag in the normal record) is fixed when the
			// scene is prepared: only triangles that emitted then change radiance.
			if (shade[3 * i + 2].w != 0.0f) {
				float4 e = shade[3 * i + 1];
				e.x = fmaxf(emission[3 * i], 0.0f);
				e.y = fmaxf(emission[3 * i + 1], 0.0f);
				e.z = fmaxf(emission[3 * i + 2], 0.0f);
				shade[3 * i + 1] = e;
			}
		}
	}
}

cudaError_t launch_set_materials(float4 *shade, int n, const float *albedo, const float *emission, cudaStream_t st) {
	if (n <= 0)
		return cudaSuccess;
	const int blocks = (n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8;
	k_set_materials<<<blocks, 256, 0, st>>>(shade, n, albedo, emission);
	return cudaGetLastError();
}

} // namespace rnb
