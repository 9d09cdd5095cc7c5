// Path-replay adjoint of the physical estimator (path replay backpropagation,
// Vicini, Speierer, Jakob 2021): d(loss)/d(per-triangle albedo) and
// d(loss)/d(per-triangle emitted radiance) with O(1) memory per path.
//
// A path is identified by its counter-based RNG key (pixel, sample), so the
// adjoint regenerates it instead of storing it. At every vertex k with albedo
// a_k the derivative of the path's radiance C is
//     g * (N_k * dlog f_k(light)/da_k + (C - P_k) * dlog w_k/da_k)
// added to dL/da[tri_k], where g = dL/dI(pixel) / spp, N_k is the vertex's
// next-event term, P_k the radiance gathered up to and including vertex k, and
// w_k the continuation weight (albedo for Lambert, F G2/G1 for GGX). Emission
// terms E add g * E / Le to dL/dLe of their emitter. Roulette probabilities are
// treated as constants.
//
// The next-event and emission terms are known at their vertex. The continuation
// terms need C, which is known when the path ends, so each thread keeps the
// (triangle, P_k, dlog w_k) of its path's first kAdjList continuation vertices
// in local memory and adds them then: one trace per sample. Only a path longer
// than that is traced a second time (its replay adds the remaining continuation
// terms). Work is one (pixel, sample) per lane, handed out to persistent warps
// in batches of 32 in sample-major order. Small scenes accumulate in shared
// memory and flush once per block; large scenes add straight to global memory.
#include "adjoint.hpp"

namespace rnb {

namespace {

constexpr int kAdjList = 8;

__device__ __forceinline__ int find_view(const AdjView *v, int n, unsigned item) {
	int lo = 0, hi = n - 1;
	while (lo < hi) {
		const int mid = (lo + hi + 1) >> 1;
		if (v[mid].item_base <= item)
			lo = mid;
		else
			hi = mid - 1;
	}
	return lo;
}

template <bool kShared>
__device__ __forceinline__ void add3(float *gbuf, float *sbuf, int tri, F3 v) {
	add_grad3(kShared ? sbuf + 3 * tri : gbuf + 3 * static_cast<size_t>(tri), v);
}

struct AdjEntry {
	int tri;
	F3 P;    // radiance gathered up to and including the vertex
	F3 dlog; // d log(continuation weight) / d albedo
};

// The radiance of the path traced from ps, with its vertices' immediate
// derivative terms (emission, next-event) added; the first kAdjList
// continuation vertices are kept in list. Returns the number of continuation
// vertices of the path.
template <bool kShared>
__device__ __forceinline__ int adjoint_path(const PhysScene &sc, const PhysSettings &st, PathState &ps, F3 g,
                                            float *d_alb, float *d_em, float *s_alb, float *s_em, AdjEntry *list,
                                            int &err) {
	F3 P = f3(0.0f, 0.0f, 0.0f);
	int nk = 0;
	for (;;) {
		const RayPre r = make_ray(ps.o.x, ps.o.y, ps.o.z, ps.d.x, ps.d.y, ps.d.z);
		const HitRec h = trace_closest_best<kOrderReference>(sc.sv, r, ps.ignore, err);
		ShadowReq sr;
		VertexGrad vg;
		const bool alive = shade_vertex_t<true>(sc, st, ps, h, sr, &vg);
		if (h.idx < 0) // an escaping ray gathers the environment (shade_vertex_t's miss term)
			P = P + ps.beta * f3(st.env[0], st.env[1], st.env[2]);
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
		if (nk < kAdjList)
			list[nk] = AdjEntry{vg.tri, P, vg.cont_dlog};
		nk++;
	}
	ps.L = P;
	return nk;
}

// Replay of a path longer than the list: continuation terms of vertices >= kAdjList.
template <bool kShared>
__device__ __forceinline__ void adjoint_replay_tail(const PhysScene &sc, const PhysSettings &st, PathState ps, F3 g,
                                                    F3 C, float *d_alb, float *s_alb, int &err) {
	F3 P = f3(0.0f, 0.0f, 0.0f);
	int k = 0;
	for (;;) {
		const RayPre r = make_ray(ps.o.x, ps.o.y, ps.o.z, ps.d.x, ps.d.y, ps.d.z);
		const HitRec h = trace_closest_best<kOrderReference>(sc.sv, r, ps.ignore, err);
		ShadowReq sr;
		VertexGrad vg;
		const bool alive = shade_vertex_t<true>(sc, st, ps, h, sr, &vg);
		if (h.idx < 0)
			P = P + ps.beta * f3(st.env[0], st.env[1], st.env[2]);
		if (vg.hit_emitter >= 0)
			P = P + vg.emit;
		if (sr.valid) {
			const RayPre rs = make_ray(sr.o.x, sr.o.y, sr.o.z, sr.d.x, sr.d.y, sr.d.z);
			if (!trace_any_best(sc.sv, rs, sr.tmax, sr.ignore, err))
				P = P + vg.nee_contrib;
		}
		if (!alive)
			break;
		if (k >= kAdjList)
			add3<kShared>(d_alb, s_alb, vg.tri, g * (C - P) * vg.cont_dlog);
		k++;
	}
}

template <bool kShared>
__global__ void __launch_bounds__(128, 8) k_adjoint(PhysScene sc, const AdjView *__restrict__ views, int n_views,
                                                 unsigned total_items, float *__restrict__ d_alb,
                                                 float *__restrict__ d_em, int n_tris, unsigned *counter,
                                                 int *status) {
	extern __shared__ float smem[];
	float *s_alb = smem;
	float *s_em = smem + 3 * n_tris;
	if (kShared) {
		for (int i = threadIdx.x; i < 6 * n_tris; i += blockDim.x)
			smem[i] = 0.0f;
		__syncthreads();
	}
	int err = 0;
	const int lane = threadIdx.x & 31;
	AdjEntry list[kAdjList];
	for (;;) {
		unsigned base = 0;
		if (lane == 0)
			base = atomicAdd(counter, 32u);
		base = __shfl_sync(0xffffffffu, base, 0);
		if (base >= total_items)
			break;
		const unsigned item = base + static_cast<unsigned>(lane);
		if (item >= total_items)
			continue;
		const AdjView &view = views[find_view(views, n_views, item)];
		const unsigned rel = item - view.item_base;
		const unsigned s = rel / static_cast<unsigned>(view.n_pix);
		const unsigned pix = rel - s * static_cast<unsigned>(view.n_pix);
		const float inv = 1.0f / static_cast<float>(view.st.spp); // spp > 0: the view has items
		const F3 g = f3(view.dimg[3 * pix] * inv, view.dimg[3 * pix + 1] * inv, view.dimg[3 * pix + 2] * inv);
		if (g.x == 0.0f && g.y == 0.0f && g.z == 0.0f)
			continue;
		const uint32_t sample = view.st.sample_offset + s;
		PathState ps = camera_path(view.cam, view.st, pix, sample);
		const int nk = adjoint_path<kShared>(sc, view.st, ps, g, d_alb, d_em, s_alb, s_em, list, err);
		const F3 C = ps.L;
		const int nl = nk < kAdjList ? nk : kAdjList;
		for (int e = 0; e < nl; e++)
			add3<kShared>(d_alb, s_alb, list[e].tri, g * (C - list[e].P) * list[e].dlog);
		if (nk > kAdjList)
			adjoint_replay_tail<kShared>(sc, view.st, camera_path(view.cam, view.st, pix, sample), g, C, d_alb,
			                             s_alb, err);
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

cudaError_t launch_adjoint(const PhysScene &sc, const AdjView *d_views, int n_views, unsigned total_items,
                           float *d_alb, float *d_em, int n_tris, unsigned *counter, int *status, cudaStream_t st) {
	if (total_items == 0)
		return cudaSuccess;
	cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned), st);
	if (e != cudaSuccess)
		return e;
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
	const unsigned need = (total_items + 127) / 128;
	if (static_cast<unsigned>(blocks) > need)
		blocks = static_cast<int>(need);
	if (shared)
		k_adjoint<true><<<blocks, 128, smem, st>>>(sc, d_views, n_views, total_items, d_alb, d_em, n_tris, counter,
		                                           status);
	else
		k_adjoint<false><<<blocks, 128, 0, st>>>(sc, d_views, n_views, total_items, d_alb, d_em, n_tris, counter,
		                                         status);
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
