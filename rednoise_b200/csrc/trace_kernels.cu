// Batched ray queries: one thread per ray over the flattened reference BVH.
#include "scene_impl.hpp"

namespace rnb {

template <int kOrder>
__global__ void __launch_bounds__(128) k_trace_closest(SceneView s, int n, const float *__restrict__ o,
                                                       const float *__restrict__ d, const int *__restrict__ ignore,
                                                       int *__restrict__ tri, float *__restrict__ t,
                                                       float *__restrict__ u, float *__restrict__ v, int *err) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const RayPre r = make_ray(o[3 * i], o[3 * i + 1], o[3 * i + 2], d[3 * i], d[3 * i + 1], d[3 * i + 2]);
	int e = 0;
	const HitRec h = trace_closest_best<kOrder>(s, r, ignore ? ignore[i] : -1, e);
	if (e)
		atomicOr(err, 1);
	tri[i] = h.idx;
	if (t)
		t[i] = h.t;
	if (u)
		u[i] = h.u;
	if (v)
		v[i] = h.v;
}

__global__ void __launch_bounds__(128) k_trace_any(SceneView s, int n, const float *__restrict__ o,
                                                   const float *__restrict__ d, const float *__restrict__ tmax,
                                                   const int *__restrict__ ignore, int *__restrict__ occ, int *err) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const RayPre r = make_ray(o[3 * i], o[3 * i + 1], o[3 * i + 2], d[3 * i], d[3 * i + 1], d[3 * i + 2]);
	int e = 0;
	const bool hit = trace_any_best(s, r, tmax[i], ignore ? ignore[i] : -1, e);
	if (e)
		atomicOr(err, 1);
	occ[i] = hit ? 1 : 0;
}

cudaError_t launch_trace_closest(const SceneView &v, int n, const float *o, const float *d, const int *ignore,
                                 int order, int *tri, float *t, float *u, float *vv, int *err, cudaStream_t st) {
	if (n <= 0)
		return cudaSuccess;
	const int bs = 128;
	if (order == kOrderNearest)
		k_trace_closest<kOrderNearest><<<ceil_div(n, bs), bs, 0, st>>>(v, n, o, d, ignore, tri, t, u, vv, err);
	else
		k_trace_closest<kOrderReference><<<ceil_div(n, bs), bs, 0, st>>>(v, n, o, d, ignore, tri, t, u, vv, err);
	return cudaGetLastError();
}

cudaError_t launch_trace_any(const SceneView &v, int n, const float *o, const float *d, const float *tmax,
                             const int *ignore, int *occ, int *err, cudaStream_t st) {
	if (n <= 0)
		return cudaSuccess;
	const int bs = 128;
	k_trace_any<<<ceil_div(n, bs), bs, 0, st>>>(v, n, o, d, tmax, ignore, occ, err);
	return cudaGetLastError();
}

} // namespace rnb
