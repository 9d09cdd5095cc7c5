// A BVH built on the GPU: the linear BVH of Karras (2012), "Maximizing Parallelism
// in the Construction of BVHs, Octrees, and k-d Trees".
//
// The reference builds its median-split tree on the host (src/BVH.cpp:6-63) and its
// closest hits are defined by that tree, so the default path keeps it. This tree is
// for callers that rebuild often (animated or edited geometry): every step is a
// data-parallel kernel over the triangles, with no host work beyond the upload.
//   1. scene bounds of the triangle centroids (a min/max reduction);
//   2. 30-bit Morton codes of the centroids, made unique as (code << 32 | index);
//   3. a radix sort of those keys;
//   4. every internal node i finds its key range and split from the longest common
//      prefixes of its neighbours' keys (Karras' construction), one thread each;
//   5. bottom-up boxes: each leaf walks to the root, and the second child to arrive
//      at a node forms that node's box (an atomic counter per node);
//   6. the nodes are written in the 2-wide device layout the traversals read.
// Leaves hold one triangle; the tree is traversed nearest-child-first with ties on
// the hit distance broken by leaf position, so its closest hits agree with the
// reference tree's except where two triangles are hit at the same distance or the
// reference's box test rejects a grazing hit.
#include <cub/cub.cuh>

#include "lbvh.hpp"

namespace rnb {

namespace {

__device__ __forceinline__ float fmin3(float a, float b, float c) { return fminf(fminf(a, b), c); }
__device__ __forceinline__ float fmax3(float a, float b, float c) { return fmaxf(fmaxf(a, b), c); }

struct Box {
	float lo[3], hi[3];
};

__global__ void k_centroid_bounds(const float *__restrict__ v9, int n, float *__restrict__ bounds) {
	// bounds: lo[3] as ordered-int atomics, hi[3]; one block-level reduction, then global atomics
	__shared__ float s_lo[3][256], s_hi[3][256];
	float lo[3] = {__int_as_float(0x7f800000), __int_as_float(0x7f800000), __int_as_float(0x7f800000)};
	float hi[3] = {-lo[0], -lo[0], -lo[0]};
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const float *t = v9 + 9 * static_cast<size_t>(i);
		for (int a = 0; a < 3; a++) {
			const float c = (t[a] + t[3 + a] + t[6 + a]) * (1.0f / 3.0f);
			lo[a] = fminf(lo[a], c);
			hi[a] = fmaxf(hi[a], c);
		}
	}
	for (int a = 0; a < 3; a++) {
		s_lo[a][threadIdx.x] = lo[a];
		s_hi[a][threadIdx.x] = hi[a];
	}
	__syncthreads();
	for (int w = blockDim.x / 2; w > 0; w >>= 1) {
		if (threadIdx.x < w)
			for (int a = 0; a < 3; a++) {
				s_lo[a][threadIdx.x] = fminf(s_lo[a][threadIdx.x], s_lo[a][threadIdx.x + w]);
				s_hi[a][threadIdx.x] = fmaxf(s_hi[a][threadIdx.x], s_hi[a][threadIdx.x + w]);
			}
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		// Floats compare like their bit patterns once the sign bit is flipped for
		// negatives; atomicMin/Max on the transformed unsigned values.
		auto key = [](float f) {
			const unsigned u = __float_as_uint(f);
			return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
		};
		unsigned *b = reinterpret_cast<unsigned *>(bounds);
		for (int a = 0; a < 3; a++) {
			atomicMin(b + a, key(s_lo[a][0]));
			atomicMax(b + 3 + a, key(s_hi[a][0]));
		}
	}
}

__device__ __forceinline__ float from_key(unsigned k) {
	return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// 10 bits per axis, interleaved (x highest).
__device__ __forceinline__ unsigned spread10(unsigned v) {
	v &= 0x3ffu;
	v = (v | (v << 16)) & 0x030000ffu;
	v = (v | (v << 8)) & 0x0300f00fu;
	v = (v | (v << 4)) & 0x030c30c3u;
	v = (v | (v << 2)) & 0x09249249u;
	return v;
}

__global__ void k_morton(const float *__restrict__ v9, int n, const float *__restrict__ bounds,
                         unsigned long long *__restrict__ keys, int *__restrict__ idx) {
	const unsigned *b = reinterpret_cast<const unsigned *>(bounds);
	float lo[3], ext[3];
	for (int a = 0; a < 3; a++) {
		lo[a] = from_key(b[a]);
		const float e = from_key(b[3 + a]) - lo[a];
		ext[a] = e > 0.0f ? 1024.0f / e : 0.0f;
	}
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const float *t = v9 + 9 * static_cast<size_t>(i);
		unsigned q[3];
		for (int a = 0; a < 3; a++) {
			const float c = (t[a] + t[3 + a] + t[6 + a]) * (1.0f / 3.0f);
			q[a] = static_cast<unsigned>(fminf(fmaxf((c - lo[a]) * ext[a], 0.0f), 1023.0f));
		}
		const unsigned code = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
		keys[i] = (static_cast<unsigned long long>(code) << 32) | static_cast<unsigned>(i);
		idx[i] = i;
	}
}

// Longest common prefix of keys i and j (-1 outside [0, n)).
__device__ __forceinline__ int delta(const unsigned long long *k, int n, int i, int j) {
	if (j < 0 || j >= n)
		return -1;
	return __clzll(k[i] ^ k[j]);
}

// Internal node i of Karras' tree: its children. Child refs: internal node index,
// or -(leaf + 1) for a leaf.
__global__ void k_karras(const unsigned long long *__restrict__ k, int n, int *__restrict__ left,
                         int *__restrict__ right, int *__restrict__ parent_int, int *__restrict__ parent_leaf) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n - 1)
		return;
	const int d = (delta(k, n, i, i + 1) - delta(k, n, i, i - 1)) >= 0 ? 1 : -1;
	const int dmin = delta(k, n, i, i - d);
	int lmax = 2;
	while (delta(k, n, i, i + lmax * d) > dmin)
		lmax <<= 1;
	int l = 0;
	for (int t = lmax >> 1; t >= 1; t >>= 1)
		if (delta(k, n, i, i + (l + t) * d) > dmin)
			l += t;
	const int j = i + l * d;
	const int dnode = delta(k, n, i, j);
	int s = 0;
	for (int t = (l + 1) >> 1;; t = (t + 1) >> 1) {
		if (delta(k, n, i, i + (s + t) * d) > dnode)
			s += t;
		if (t == 1)
			break;
	}
	const int gamma = i + s * d + (d < 0 ? -1 : 0);
	const int lo = i < j ? i : j, hi = i < j ? j : i;
	const int lc = lo == gamma ? -(gamma + 1) : gamma;
	const int rc = hi == gamma + 1 ? -(gamma + 2) : gamma + 1;
	left[i] = lc;
	right[i] = rc;
	if (lc < 0)
		parent_leaf[-lc - 1] = i;
	else
		parent_int[lc] = i;
	if (rc < 0)
		parent_leaf[-rc - 1] = i;
	else
		parent_int[rc] = i;
}

__device__ __forceinline__ Box load_box_cg(const Box *p) {
	const float *f = reinterpret_cast<const float *>(p);
	Box b;
	for (int a = 0; a < 3; a++) {
		b.lo[a] = __ldcg(f + a);
		b.hi[a] = __ldcg(f + 3 + a);
	}
	return b;
}

// Leaf boxes, the leaf-ordered triangle records, then boxes up the tree.
__global__ void k_refit(const float *__restrict__ v9, const int *__restrict__ order, int n,
                        const int *__restrict__ left, const int *__restrict__ right,
                        const int *__restrict__ parent_int, const int *__restrict__ parent_leaf,
                        unsigned *__restrict__ arrived, Box *__restrict__ leaf_box, Box *__restrict__ node_box,
                        float4 *__restrict__ tris) {
	const int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n)
		return;
	const int ti = order[p];
	const float *t = v9 + 9 * static_cast<size_t>(ti);
	Box b;
	for (int a = 0; a < 3; a++) {
		b.lo[a] = fmin3(t[a], t[3 + a], t[6 + a]);
		b.hi[a] = fmax3(t[a], t[3 + a], t[6 + a]);
	}
	leaf_box[p] = b;
	// v0, e0 = v1 - v0, e1 = v2 - v0 (IEEE subtraction, as the host layout); rank = leaf position
	tris[3 * static_cast<size_t>(p)] = make_float4(t[0], t[1], t[2], __int_as_float(ti));
	tris[3 * static_cast<size_t>(p) + 1] =
	    make_float4(__fsub_rn(t[3], t[0]), __fsub_rn(t[4], t[1]), __fsub_rn(t[5], t[2]), __int_as_float(p));
	tris[3 * static_cast<size_t>(p) + 2] =
	    make_float4(__fsub_rn(t[6], t[0]), __fsub_rn(t[7], t[1]), __fsub_rn(t[8], t[2]), 0.0f);
	if (n == 1)
		return;
	int node = parent_leaf[p];
	while (node >= 0) {
		__threadfence();
		if (atomicAdd(arrived + node, 1u) == 0)
			return; // the sibling's thread finishes this node
		__threadfence();
		const int lc = left[node], rc = right[node];
		// the sibling's box was written by another thread: read past L1
		const Box bl = load_box_cg(lc < 0 ? leaf_box + (-lc - 1) : node_box + lc);
		const Box br = load_box_cg(rc < 0 ? leaf_box + (-rc - 1) : node_box + rc);
		Box m;
		for (int a = 0; a < 3; a++) {
			m.lo[a] = fminf(bl.lo[a], br.lo[a]);
			m.hi[a] = fmaxf(bl.hi[a], br.hi[a]);
		}
		node_box[node] = m;
		node = node == 0 ? -1 : parent_int[node];
	}
}

// Depth of every leaf (root = 1), reduced to the maximum.
__global__ void k_depth(int n, const int *__restrict__ parent_int, const int *__restrict__ parent_leaf,
                        int *__restrict__ depth_out) {
	const int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n)
		return;
	int depth = 1;
	for (int node = n > 1 ? parent_leaf[p] : -1; node >= 0; node = node == 0 ? -1 : parent_int[node])
		depth++;
	atomicMax(depth_out, depth);
}

__device__ __forceinline__ int leaf_ref_of(int leaf) { return ~((leaf << 3) | 1); }

// The 2-wide device layout: per internal node both children's boxes and refs.
__global__ void k_lbvh_nodes(int n, const int *__restrict__ left, const int *__restrict__ right,
                             const Box *__restrict__ leaf_box, const Box *__restrict__ node_box,
                             float4 *__restrict__ nodes) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n - 1)
		return;
	const int lc = left[i], rc = right[i];
	const Box L = lc < 0 ? leaf_box[-lc - 1] : node_box[lc];
	const Box R = rc < 0 ? leaf_box[-rc - 1] : node_box[rc];
	float4 *o = nodes + 4 * static_cast<size_t>(i);
	o[0] = make_float4(L.lo[0], L.hi[0], L.lo[1], L.hi[1]);
	o[1] = make_float4(R.lo[0], R.hi[0], R.lo[1], R.hi[1]);
	o[2] = make_float4(L.lo[2], L.hi[2], R.lo[2], R.hi[2]);
	o[3] = make_float4(__int_as_float(lc < 0 ? leaf_ref_of(-lc - 1) : lc),
	                   __int_as_float(rc < 0 ? leaf_ref_of(-rc - 1) : rc), 0.0f, 0.0f);
}

inline size_t a256(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }
inline int blocks_for(long n, int bs) { return static_cast<int>((n + bs - 1) / bs); }

} // namespace

size_t lbvh_scratch_bytes(int n) {
	size_t sort_bytes = 0;
	cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, static_cast<unsigned long long *>(nullptr),
	                                static_cast<unsigned long long *>(nullptr), static_cast<int *>(nullptr),
	                                static_cast<int *>(nullptr), n);
	const size_t nn = static_cast<size_t>(n);
	return a256(24) + 2 * a256(nn * 8) + 2 * a256(nn * 4) + 4 * a256(nn * 4) + a256(nn * 4) + a256(nn * sizeof(Box)) +
	       a256(nn * sizeof(Box)) + a256(sort_bytes) + a256(16) + 1024;
}

cudaError_t lbvh_build(const float *d_v9, int n, void *scratch, size_t scratch_bytes, float4 *d_nodes,
                       float4 *d_tris, LbvhResult &res, cudaStream_t st) {
	if (n <= 0)
		return cudaErrorInvalidValue;
	const size_t nn = static_cast<size_t>(n);
	char *b = static_cast<char *>(scratch);
	auto take = [&b](size_t bytes) {
		char *p = b;
		b += a256(bytes);
		return p;
	};
	float *d_bounds = reinterpret_cast<float *>(take(24));
	unsigned long long *k0 = reinterpret_cast<unsigned long long *>(take(nn * 8));
	unsigned long long *k1 = reinterpret_cast<unsigned long long *>(take(nn * 8));
	int *i0 = reinterpret_cast<int *>(take(nn * 4));
	int *i1 = reinterpret_cast<int *>(take(nn * 4));
	int *left = reinterpret_cast<int *>(take(nn * 4));
	int *right = reinterpret_cast<int *>(take(nn * 4));
	int *par_int = reinterpret_cast<int *>(take(nn * 4));
	int *par_leaf = reinterpret_cast<int *>(take(nn * 4));
	unsigned *arrived = reinterpret_cast<unsigned *>(take(nn * 4));
	Box *leaf_box = reinterpret_cast<Box *>(take(nn * sizeof(Box)));
	Box *node_box = reinterpret_cast<Box *>(take(nn * sizeof(Box)));
	int *d_depth = reinterpret_cast<int *>(take(16));
	void *tmp = take(0);
	const size_t used = static_cast<size_t>(b - static_cast<char *>(scratch));
	if (used > scratch_bytes)
		return cudaErrorInvalidValue;
	size_t tmp_bytes = scratch_bytes - used;

	// bounds: lo keys start at +max (0xffffffff), hi keys at 0
	cudaError_t e = cudaMemsetAsync(d_bounds, 0xff, 12, st);
	if (e == cudaSuccess)
		e = cudaMemsetAsync(reinterpret_cast<char *>(d_bounds) + 12, 0, 12, st);
	if (e == cudaSuccess)
		e = cudaMemsetAsync(arrived, 0, nn * 4, st);
	if (e == cudaSuccess)
		e = cudaMemsetAsync(d_depth, 0, 4, st);
	if (e != cudaSuccess)
		return e;
	const int gb = blocks_for(n, 256) < 148 * 8 ? blocks_for(n, 256) : 148 * 8;
	k_centroid_bounds<<<gb, 256, 0, st>>>(d_v9, n, d_bounds);
	k_morton<<<gb, 256, 0, st>>>(d_v9, n, d_bounds, k0, i0);
	e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, k0, k1, i0, i1, n, 0, 64, st);
	if (e != cudaSuccess)
		return e;
	if (n > 1)
		k_karras<<<blocks_for(n - 1, 256), 256, 0, st>>>(k1, n, left, right, par_int, par_leaf);
	k_refit<<<blocks_for(n, 256), 256, 0, st>>>(d_v9, i1, n, left, right, par_int, par_leaf, arrived, leaf_box,
	                                           node_box, d_tris);
	k_depth<<<blocks_for(n, 256), 256, 0, st>>>(n, par_int, par_leaf, d_depth);
	if (n > 1)
		k_lbvh_nodes<<<blocks_for(n - 1, 256), 256, 0, st>>>(n, left, right, leaf_box, node_box, d_nodes);
	e = cudaGetLastError();
	if (e != cudaSuccess)
		return e;
	// root box and depth back to the host
	Box root;
	e = cudaMemcpyAsync(&root, n > 1 ? node_box : leaf_box, sizeof(Box), cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(&res.depth, d_depth, 4, cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(st);
	if (e != cudaSuccess)
		return e;
	for (int a = 0; a < 3; a++) {
		res.root_lo[a] = root.lo[a];
		res.root_hi[a] = root.hi[a];
	}
	res.root_ref = n > 1 ? 0 : ~((0 << 3) | 1);
	res.internal_nodes = n - 1;
	if (n == 1)
		res.depth = 1;
	return cudaSuccess;
}

} // namespace rnb
