// Wavefront integrator kernels (see wavefront.cuh).
#include "wavefront.cuh"
#include "pixel_tiles.cuh"

namespace rnb {

namespace {

__device__ __forceinline__ unsigned lanemask_lt() {
	unsigned m;
	asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
	return m;
}

// Warp-aggregated append: one atomicAdd per warp for all lanes with pred set.
__device__ __forceinline__ unsigned warp_append(unsigned *ctr, bool pred) {
	const unsigned active = __activemask();
	const unsigned ballot = __ballot_sync(active, pred);
	const int leader = __ffs(active) - 1;
	const int lane = threadIdx.x & 31;
	unsigned base = 0;
	if (lane == leader && ballot)
		base = atomicAdd(ctr, static_cast<unsigned>(__popc(ballot)));
	base = __shfl_sync(active, base, leader);
	return base + static_cast<unsigned>(__popc(ballot & lanemask_lt()));
}

// Last entry of a sorted base table that is <= x.
__device__ __forceinline__ int find_base(const int *bases, int n, int x) {
	int lo = 0, hi = n - 1;
	while (lo < hi) {
		const int mid = (lo + hi + 1) >> 1;
		if (bases[mid] <= x)
			lo = mid;
		else
			hi = mid - 1;
	}
	return lo;
}

__global__ void __launch_bounds__(256) k_wf_camera(const WfJob *__restrict__ jobs, WfPool pool, WfWave wave) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < wave.n_slots; i += gridDim.x * blockDim.x) {
		const int a = find_base(wave.bases, wave.n_jobs, i);
		const int j = wave.jobs[a];
		const WfJob &job = jobs[j];
		const int rel = i - wave.bases[a];
		const uint32_t pixel = static_cast<uint32_t>(rel % job.n_pix);
		const uint32_t sample =
		    job.st.sample_offset + static_cast<uint32_t>(wave.first_sample + rel / job.n_pix);
		const PathState ps = camera_path(job.cam, job.st, pixel, sample);
		pool.o[i] = make_float4(ps.o.x, ps.o.y, ps.o.z, __int_as_float(-1));
		pool.d[i] = make_float4(ps.d.x, ps.d.y, ps.d.z, 0.0f);
		// beta is not written: the first shading stage takes throughput 1 at bounce 0
		pool.L[i] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(j));
		pool.pixel[i] = pixel;
		pool.sample[i] = sample;
		const bool tiled = job.cam.width > 0 && job.cam.height > 0 &&
		                   static_cast<long long>(job.cam.width) * job.cam.height == job.n_pix;
		const int in_block = tiled ? static_cast<int>(tile_order(pixel, job.cam.width, job.cam.height))
		                           : static_cast<int>(pixel);
		pool.queue[0][i - static_cast<int>(pixel) + in_block] = i;
	}
	if (blockIdx.x == 0 && threadIdx.x == 0)
		pool.counters[kCntRays] = static_cast<unsigned>(wave.n_slots);
}

// Top entries of the traversal stack that the one-ray-per-lane traversal stages
// keep in shared memory, the rest in local memory (0: all in local memory). On
// the 1.31M-triangle frame with the speculative traversals, 8 and 16 entries gave
// the same closest-hit stage (103.5 ms) and the all-local stack 105.4 ms.
constexpr int kWfShortStack = 8;
constexpr size_t kWfExtendSmem = static_cast<size_t>(kWfShortStack) * 128 * sizeof(unsigned long long);
constexpr size_t kWfShadowSmem = static_cast<size_t>(kWfShortStack) * 128 * sizeof(int);

template <int kOrder>
__global__ void __launch_bounds__(128) k_wf_extend(const WfJob *__restrict__ jobs, WfPool pool, int k,
                                                   const int *__restrict__ q, int only_job, int *status) {
	const unsigned n = pool.counters[kCntRays + k];
	const int lane = threadIdx.x & 31;
	int err = 0;
	for (;;) {
		unsigned base = 0;
		if (lane == 0)
			base = atomicAdd(pool.counters + kCntFetchExt + k, 32u);
		base = __shfl_sync(0xffffffffu, base, 0);
		if (base >= n)
			break;
		const unsigned i = base + lane;
		if (i < n) {
			const int slot = q[i];
			const float4 o = pool.o[slot];
			const float4 d = pool.d[slot];
			const int j = only_job >= 0 ? only_job : __float_as_int(pool.L[slot].w);
			const RayPre r = make_ray(o.x, o.y, o.z, d.x, d.y, d.z);
			HitRec h;
			if constexpr (kWfShortStack > 0) {
				extern __shared__ unsigned long long wf_ext_stack[];
				SharedShortStack<unsigned long long, kWfShortStack> st(wf_ext_stack + threadIdx.x, blockDim.x);
				h = trace_closest_best<kOrder>(jobs[j].sc.sv, r, __float_as_int(o.w), err, st);
			} else {
				h = trace_closest_best<kOrder>(jobs[j].sc.sv, r, __float_as_int(o.w), err);
			}
			pool.hit_idx[slot] = h.idx;
			pool.hit_t[slot] = h.t;
		}
	}
	if (err)
		atomicOr(status, 1);
}

// Bins of the binning sorts. A continuation ray's bin is the Morton cell of its
// origin (point_bin, 5 bits per axis over the scene's box) refined by a 16 x 16
// octahedral cell of its direction (dir_cell); a shadow record's bin is the cell of
// its origin alone (its direction points at the light). On the 1.31M-triangle
// 1080p frame this 23-bit order, sorted in two counting passes, took the frame from
// 208 to 191 ms against a single 15-bit key (an 8 x 8 x 8 origin cell above an
// 8 x 8 direction cell); a 30-bit key (64 x 64 x 64 origin cells, 64 x 64
// direction cells) left too few rays per bin to fill a warp and gained a third as
// much. Of the single 15-bit splits, origin-major beat direction-major, and keys that
// gave either part fewer bits were slower still.
// fmaxf maps a NaN (a flat extent: 0 * inf) to cell 0
__device__ __forceinline__ unsigned quantize(float x, float cells) {
	return static_cast<unsigned>(fminf(fmaxf(x * cells, 0.0f), cells - 1.0f));
}
// 15-bit Morton cell (5 bits per axis over the scene's box) of a ray's origin.
__device__ __forceinline__ unsigned point_bin(const SceneView &sv, const F3 &o) {
	const float q[3] = {o.x, o.y, o.z};
	unsigned m = 0;
#pragma unroll
	for (int a = 0; a < 3; a++) {
		const unsigned c = quantize((q[a] - sv.root_lo[a]) * __fdividef(1.0f, sv.root_hi[a] - sv.root_lo[a]), 32.0f);
#pragma unroll
		for (int b = 0; b < 5; b++)
			m |= ((c >> b) & 1u) << (3 * b + a);
	}
	return m;
}
static_assert(kBinBits == 15, "point_bin writes 15-bit keys");
// 6-bit Morton sub-cell of a point inside its point_bin cell (the next 2 bits per axis).
__device__ __forceinline__ unsigned point_sub_cell(const SceneView &sv, const F3 &o) {
	const float q[3] = {o.x, o.y, o.z};
	unsigned m = 0;
#pragma unroll
	for (int a = 0; a < 3; a++) {
		const unsigned c = quantize((q[a] - sv.root_lo[a]) * __fdividef(1.0f, sv.root_hi[a] - sv.root_lo[a]), 128.0f);
		m |= ((c & 1u) << a) | (((c >> 1) & 1u) << (3 + a));
	}
	return m;
}

// 8-bit cell of a direction: 16 x 16 over the unit octahedron unfolded onto a square.
__device__ __forceinline__ unsigned dir_cell(const F3 &d) {
	const float inv_l1 = __fdividef(1.0f, fabsf(d.x) + fabsf(d.y) + fabsf(d.z));
	float px = d.x * inv_l1, py = d.y * inv_l1;
	if (d.z < 0.0f) { // fold the lower hemisphere onto the corners
		const float qx = (1.0f - fabsf(py)) * (px >= 0.0f ? 1.0f : -1.0f);
		const float qy = (1.0f - fabsf(px)) * (py >= 0.0f ? 1.0f : -1.0f);
		px = qx;
		py = qy;
	}
	return (quantize(0.5f * (py + 1.0f), 16.0f) << 4) | quantize(0.5f * (px + 1.0f), 16.0f);
}

// Gradient adds of one warp merged per triangle: every lane of `mask` calls this;
// lanes with `on` set add v to base[3 tri .. 3 tri + 2]. Lanes that share a triangle
// pass their values through this warp's 96 floats of shared memory (scratch) to the
// lowest of them, which adds the sum: few emitter and wall triangles take most of the
// adjoint's terms, and one atomic per triangle and warp keeps them from queueing.
__device__ __forceinline__ void add_grad3_warp(float *base, int tri, F3 v, bool on, unsigned mask, float *scratch) {
	const int lane = threadIdx.x & 31;
	const unsigned act = __ballot_sync(mask, on);
	if (on) {
		const unsigned peers = __match_any_sync(act, tri);
		scratch[lane] = v.x;
		scratch[32 + lane] = v.y;
		scratch[64 + lane] = v.z;
		__syncwarp(act);
		if (lane == __ffs(peers) - 1) {
			F3 sum = f3(0.0f, 0.0f, 0.0f);
			for (unsigned m = peers; m; m &= m - 1) {
				const int l = __ffs(m) - 1;
				sum.x += scratch[l];
				sum.y += scratch[32 + l];
				sum.z += scratch[64 + l];
			}
			add_grad3(base + 3 * static_cast<size_t>(tri), sum);
		}
		__syncwarp(act);
	}
}

// dL/d(sample radiance) of a path of job `job` through `pixel`: the mean image's
// gradient over the job's samples per pixel.
__device__ __forceinline__ F3 adj_weight(const WfJob &job, uint32_t pixel) {
	const float inv = 1.0f / static_cast<float>(job.st.spp);
	const float *gi = job.dimg + 3 * static_cast<size_t>(pixel);
	return f3(gi[0] * inv, gi[1] * inv, gi[2] * inv);
}

// kAdj: the adjoint wave's shade stage (path replay backpropagation, the same terms
// in the same arithmetic as the per-path adjoint): the previous vertex's gathered
// radiance is complete when this stage starts (its next-event term was added by the
// shadow stage), emission terms go to d_em here, next-event terms are handed to the
// shadow stage with the record, and a continuing vertex joins the slot's list.
// Seven resident blocks per SM for the primal stage: it waits on scattered loads of
// path state, and more warps in flight measured 18.3 ms (five blocks) -> 17.3 (six)
// -> 17.0 ms (eight) on the bench frame; after the first bounce's shading moved to
// slot order, seven gave 17.25 ms against eight's 17.6, nine 18.5 and ten 23.2
// (spills). Same image throughout (the translation unit is compiled without
// multiply-add contraction, so the register budget cannot change the arithmetic).
// The adjoint instantiation keeps five: it carries the gradient terms as well.
template <bool kAdj>
__global__ void __launch_bounds__(128, kAdj ? 5 : 7) k_wf_shade(const WfJob *__restrict__ jobs, WfPool pool, int k,
                                                  const int *__restrict__ q, int write_keys, int *status) {
	const unsigned n = pool.counters[kCntRays + k];
	int *__restrict__ qn = pool.queue[(k + 1) & 1];
	for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const int slot = q ? q[i] : static_cast<int>(i); // null q: every slot, in slot order
		const float4 o = pool.o[slot], d = pool.d[slot], L = pool.L[slot];
		// a camera path enters its first shading stage with throughput 1 at bounce 0
		const float4 b = k == 0 ? make_float4(1.0f, 1.0f, 1.0f, __int_as_float(0)) : pool.beta[slot];
		const int j = __float_as_int(L.w);
		const WfJob &job = jobs[j];
		PathState ps;
		ps.o = f3(o.x, o.y, o.z);
		ps.d = f3(d.x, d.y, d.z);
		ps.beta = f3(b.x, b.y, b.z);
		ps.L = f3(L.x, L.y, L.z);
		ps.prev_pdf = d.w;
		ps.ignore = __float_as_int(o.w);
		ps.bounce = __float_as_int(b.w);
		ps.pixel = pool.pixel[slot];
		ps.sample = pool.sample[slot];
		HitRec h;
		h.idx = pool.hit_idx[slot];
		h.t = pool.hit_t[slot];
		h.u = h.v = 0.0f;
		h.rank = 0;
		ShadowReq sr;
		VertexGrad vg;
		F3 g = f3(0.0f, 0.0f, 0.0f);
		int n_list = 0;
		if constexpr (kAdj) {
			g = adj_weight(job, ps.pixel);
			n_list = pool.adj_n[slot];
			if (n_list > 0)
				pool.adj_pt[static_cast<size_t>(n_list - 1) * pool.capacity + slot] = make_float4(L.x, L.y, L.z, 0.0f);
		}
		const bool alive = shade_vertex_t<kAdj>(job.sc, job.st, ps, h, sr, kAdj ? &vg : nullptr);
		if constexpr (kAdj) {
			__shared__ float agg[4 * 96];
			const bool em = vg.hit_emitter >= 0;
			add_grad3_warp(pool.d_em, em ? vg.hit_emitter : 0, em ? g * safe_div(vg.emit, vg.Le) : f3(0.0f, 0.0f, 0.0f),
			               em, __activemask(), agg + (threadIdx.x >> 5) * 96);
		}
		const unsigned si = warp_append(pool.counters + kCntShadow + k, sr.valid);
		if (kBoundsCheck && sr.valid && si >= static_cast<unsigned>(pool.capacity)) {
			atomicOr(status, 1);
			sr.valid = false;
		}
		if (sr.valid) {
			if (write_keys) {
				pool.sh_keys[si] = static_cast<uint16_t>(point_bin(job.sc.sv, sr.o));
				pool.sh_fine[si] = static_cast<uint8_t>(point_sub_cell(job.sc.sv, sr.o));
			}
			pool.sh_o[si] = make_float4(sr.o.x, sr.o.y, sr.o.z, sr.tmax);
			pool.sh_d[si] = make_float4(sr.d.x, sr.d.y, sr.d.z, __int_as_float(sr.ignore));
			pool.sh_c[si] = make_float4(sr.contrib.x, sr.contrib.y, sr.contrib.z, __int_as_float(slot));
			if constexpr (kAdj) {
				pool.sh_gdlog[si] = make_float4(vg.nee_dlog.x, vg.nee_dlog.y, vg.nee_dlog.z, __int_as_float(vg.tri));
				pool.sh_gle[si] = make_float4(vg.nee_Le.x, vg.nee_Le.y, vg.nee_Le.z, __int_as_float(vg.nee_emitter));
			}
		}
		if constexpr (kAdj) {
			if (alive) {
				if (kBoundsCheck && n_list >= pool.adj_entries) {
					atomicOr(status, 1);
				} else {
					pool.adj_dlog[static_cast<size_t>(n_list) * pool.capacity + slot] =
					    make_float4(vg.cont_dlog.x, vg.cont_dlog.y, vg.cont_dlog.z, __int_as_float(vg.tri));
					pool.adj_n[slot] = n_list + 1;
				}
			}
		}
		const unsigned ni = warp_append(pool.counters + kCntRays + k + 1, alive);
		pool.L[slot] = make_float4(ps.L.x, ps.L.y, ps.L.z, L.w);
		if (kBoundsCheck && alive && ni >= static_cast<unsigned>(pool.capacity)) {
			atomicOr(status, 1);
			continue;
		}
		if (alive) {
			qn[ni] = slot;
			if (write_keys) {
				pool.keys[ni] = static_cast<uint16_t>(point_bin(job.sc.sv, ps.o));
				pool.fine[ni] = static_cast<uint8_t>(dir_cell(ps.d));
			}
			pool.o[slot] = make_float4(ps.o.x, ps.o.y, ps.o.z, __int_as_float(ps.ignore));
			pool.d[slot] = make_float4(ps.d.x, ps.d.y, ps.d.z, ps.prev_pdf);
			pool.beta[slot] = make_float4(ps.beta.x, ps.beta.y, ps.beta.z, __int_as_float(ps.bounce));
		}
	}
}

// kAdj: an unoccluded record also adds its next-event terms to d_alb and d_em.
template <bool kAdj>
__global__ void __launch_bounds__(128) k_wf_shadow(const WfJob *__restrict__ jobs, WfPool pool, int k, int only_job,
                                                   const int *__restrict__ order, int *status) {
	const unsigned n = pool.counters[kCntShadow + k];
	const int lane = threadIdx.x & 31;
	int err = 0;
	for (;;) {
		unsigned base = 0;
		if (lane == 0)
			base = atomicAdd(pool.counters + kCntFetchSh + k, 32u);
		base = __shfl_sync(0xffffffffu, base, 0);
		if (base >= n)
			break;
		const unsigned q = base + lane;
		// kAdj: this lane's next-event gradient terms, added by the whole warp below
		bool g_on = false;
		int g_tri = 0, g_em = 0;
		F3 g_alb_v = f3(0.0f, 0.0f, 0.0f), g_em_v = f3(0.0f, 0.0f, 0.0f);
		if (q < n) {
			const unsigned i = order ? static_cast<unsigned>(order[q]) : q;
			const float4 so = pool.sh_o[i], sd = pool.sh_d[i];
			const float4 sc = pool.sh_c[i];
			const int slot = __float_as_int(sc.w);
			const int j = only_job >= 0 ? only_job : __float_as_int(pool.L[slot].w);
			const RayPre r = make_ray(so.x, so.y, so.z, sd.x, sd.y, sd.z);
			bool occluded;
			if constexpr (kWfShortStack > 0) {
				extern __shared__ int wf_sh_stack[];
				SharedShortStack<int, kWfShortStack> st(wf_sh_stack + threadIdx.x, blockDim.x);
				occluded = trace_any_best(jobs[j].sc.sv, r, so.w, __float_as_int(sd.w), err, st);
			} else {
				occluded = trace_any_best(jobs[j].sc.sv, r, so.w, __float_as_int(sd.w), err);
			}
			if (!occluded) {
				float4 L = pool.L[slot];
				L.x += sc.x;
				L.y += sc.y;
				L.z += sc.z;
				pool.L[slot] = L;
				if constexpr (kAdj) {
					const F3 g = adj_weight(jobs[j], pool.pixel[slot]);
					const float4 gd = pool.sh_gdlog[i], gl = pool.sh_gle[i];
					const F3 c = f3(sc.x, sc.y, sc.z);
					g_on = true;
					g_tri = __float_as_int(gd.w);
					g_em = __float_as_int(gl.w);
					g_alb_v = g * c * f3(gd.x, gd.y, gd.z);
					g_em_v = g * safe_div(c, f3(gl.x, gl.y, gl.z));
				}
			}
		}
		if constexpr (kAdj) {
			__shared__ float agg[4 * 96];
			float *scratch = agg + (threadIdx.x >> 5) * 96;
			add_grad3_warp(pool.d_alb, g_tri, g_alb_v, g_on, 0xffffffffu, scratch);
			add_grad3_warp(pool.d_em, g_em, g_em_v, g_on, 0xffffffffu, scratch);
		}
	}
	if (err)
		atomicOr(status, 1);
}

// Persistent traversal with per-lane ray replacement: a lane whose ray finished
// takes the next queued ray at the following step, so warps stay full while the
// queue lasts (closest hits for the extend stage, any hits for shadow records).
template <bool kAny>
__global__ void __launch_bounds__(128) k_wf_trace_dyn(const WfJob *__restrict__ jobs, WfPool pool, int k,
                                                      const int *__restrict__ q, int only_job, int *status) {
	const unsigned n = pool.counters[(kAny ? kCntShadow : kCntRays) + k];
	unsigned *fetch = pool.counters + (kAny ? kCntFetchSh : kCntFetchExt) + k;
	const int lane = threadIdx.x & 31;
	int err = 0;
	TravState ts;
	const WfJob *jb = nullptr;
	int slot = -1;
	unsigned rec = 0;
	bool active = false, exhausted = false;
	for (;;) {
		const unsigned idle = __ballot_sync(0xffffffffu, !active);
		if (idle && !exhausted) {
			unsigned base = 0;
			if (lane == 0)
				base = atomicAdd(fetch, static_cast<unsigned>(__popc(idle)));
			base = __shfl_sync(0xffffffffu, base, 0);
			if (base + static_cast<unsigned>(__popc(idle)) >= n)
				exhausted = true;
			if (!active) {
				const unsigned i = base + static_cast<unsigned>(__popc(idle & lanemask_lt()));
				if (i < n) {
					RayPre r;
					float tmax = 0.0f;
					int ignore;
					if (kAny) {
						const float4 so = pool.sh_o[i], sd = pool.sh_d[i];
						rec = i;
						slot = __float_as_int(pool.sh_c[i].w);
						r = make_ray(so.x, so.y, so.z, sd.x, sd.y, sd.z);
						tmax = so.w;
						ignore = __float_as_int(sd.w);
					} else {
						slot = q[i];
						const float4 o = pool.o[slot], d = pool.d[slot];
						r = make_ray(o.x, o.y, o.z, d.x, d.y, d.z);
						ignore = __float_as_int(o.w);
					}
					jb = jobs + (only_job >= 0 ? only_job : __float_as_int(pool.L[slot].w));
					if (jb->sc.sv.nodes4 && finite_inverse(r)) {
						trav_begin<kAny>(ts, jb->sc.sv, r, tmax, ignore);
						active = true;
					} else if (kAny) { // rays with an infinite 1/d component: 2-wide path at once
						if (!trace_any(jb->sc.sv, r, tmax, ignore, err)) {
							const float4 c = pool.sh_c[i];
							float4 L = pool.L[slot];
							L.x += c.x;
							L.y += c.y;
							L.z += c.z;
							pool.L[slot] = L;
						}
					} else {
						const HitRec h = trace_closest<kOrderReference>(jb->sc.sv, r, ignore, err);
						pool.hit_idx[slot] = h.idx;
						pool.hit_t[slot] = h.t;
					}
				}
			}
		}
		if (!__any_sync(0xffffffffu, active) && exhausted)
			break;
		if (active && !trav_step<kAny>(ts, jb->sc.sv, err)) {
			active = false;
			if (kAny) {
				if (!ts.hit_any) {
					const float4 c = pool.sh_c[rec];
					float4 L = pool.L[slot];
					L.x += c.x;
					L.y += c.y;
					L.z += c.z;
					pool.L[slot] = L;
				}
			} else {
				pool.hit_idx[slot] = ts.h.idx;
				pool.hit_t[slot] = ts.h.t;
			}
		}
		if (err) // a corrupt tree: stop this warp's lanes from looping on it
			active = false;
	}
	if (err)
		atomicOr(status, 1);
}

// Binning sorts of the closest-hit and shadow queues of bounce k (counting sorts on
// the keys the shade stage wrote). A counting sort of `*count` items by 15-bit key:
// out[position] = items[i], or i when items is null; with fine set, fine_out[position]
// = fine[i] as well. Each of `grid` blocks (1024 threads, a kBins-word histogram in
// dynamic shared memory) owns one contiguous chunk of the items:
//   count:   the chunk's histogram, written as row `block` of hist (block-major);
//   colscan: per bin, the exclusive prefix of its row entries over the blocks (in
//            place) and the bin's total, into bins[0, kBins);
//   scatter: every block scans the bin totals into exclusive bin starts on its own
//            (block 0 also stores them in bins[kBins, 2 kBins)), then places its
//            items from start[key] + hist[b][key] on, with shared-memory atomics only.
// No global atomics: a block's share of every bin is known before it writes. Keys
// are masked to kBins so every shared-memory index is in range.
struct BinSrc {
	const uint16_t *keys;
	const unsigned *count;
	const int *items;
	int *out;
	const uint8_t *fine;
	uint8_t *fine_out;
};

// The items [c0, c1) of block `blk` of `nblk` (the same split in count and scatter).
__device__ __forceinline__ void bin_chunk(unsigned n, unsigned blk, unsigned nblk, unsigned &c0, unsigned &c1) {
	const unsigned per = (n + nblk - 1) / nblk;
	c0 = min(n, blk * per);
	c1 = min(n, c0 + per);
}

__global__ void __launch_bounds__(1024) k_wf_bin_count(BinSrc src, unsigned *hist) {
	extern __shared__ __align__(16) unsigned h[];
	for (int b = threadIdx.x; b < kBins; b += blockDim.x)
		h[b] = 0;
	__syncthreads();
	unsigned c0, c1;
	bin_chunk(*src.count, blockIdx.x, gridDim.x, c0, c1);
	for (unsigned i = c0 + threadIdx.x; i < c1; i += blockDim.x)
		atomicAdd(&h[src.keys[i] & (kBins - 1)], 1u);
	__syncthreads();
	uint4 *row = reinterpret_cast<uint4 *>(hist + static_cast<size_t>(blockIdx.x) * kBins);
	const uint4 *hv = reinterpret_cast<const uint4 *>(h);
	for (int b = threadIdx.x; b < kBins / 4; b += blockDim.x)
		row[b] = hv[b];
}

// kColSplit consecutive lanes per bin, each walking one stretch of the blocks' rows
// (eight loads in flight), joined by a shuffle scan across the stretches.
constexpr int kColScanThreads = 256;
constexpr int kColSplit = 4;
static_assert(kBins * kColSplit % kColScanThreads == 0, "k_wf_bin_colscan covers the bins exactly");
static_assert(32 % kColSplit == 0, "a bin's lanes share a warp");
__global__ void __launch_bounds__(kColScanThreads) k_wf_bin_colscan(unsigned *hist, int blocks, unsigned *bins) {
	const int g = blockIdx.x * blockDim.x + threadIdx.x;
	const int b = g / kColSplit, part = g % kColSplit;
	const int per = (blocks + kColSplit - 1) / kColSplit;
	const int k0 = min(blocks, part * per), k1 = min(blocks, k0 + per);
	unsigned sum = 0;
	int k = k0;
	for (; k + 8 <= k1; k += 8) {
#pragma unroll
		for (int j = 0; j < 8; j++)
			sum += hist[static_cast<size_t>(k + j) * kBins + b];
	}
	for (; k < k1; k++)
		sum += hist[static_cast<size_t>(k) * kBins + b];
	unsigned x = sum;
	for (int o = 1; o < kColSplit; o <<= 1) {
		const unsigned y = __shfl_up_sync(0xffffffffu, x, o, kColSplit);
		if (part >= o)
			x += y;
	}
	const unsigned total = __shfl_sync(0xffffffffu, x, kColSplit - 1, kColSplit);
	unsigned run = x - sum;
	k = k0;
	for (; k + 8 <= k1; k += 8) {
		unsigned c[8];
#pragma unroll
		for (int j = 0; j < 8; j++)
			c[j] = hist[static_cast<size_t>(k + j) * kBins + b];
#pragma unroll
		for (int j = 0; j < 8; j++) {
			hist[static_cast<size_t>(k + j) * kBins + b] = run;
			run += c[j];
		}
	}
	for (; k < k1; k++) {
		const unsigned c = hist[static_cast<size_t>(k) * kBins + b];
		hist[static_cast<size_t>(k) * kBins + b] = run;
		run += c;
	}
	if (part == 0)
		bins[b] = total;
}

// Exclusive scan of the kBins bin totals into shared memory, by one block of 1024
// threads (32 consecutive bins each); every scatter block runs it on its own copy.
constexpr int kScanThreads = 1024;
constexpr int kBinsPerThread = kBins / kScanThreads;
static_assert(kBins == kScanThreads * 32, "block_scan_bins gives each thread 8 uint4 of bins");
__device__ __forceinline__ void block_scan_bins(const unsigned *totals, unsigned *h, unsigned *warp_sum) {
	const int t = threadIdx.x;
	const uint4 *tv = reinterpret_cast<const uint4 *>(totals) + t * (kBinsPerThread / 4);
	uint4 v[kBinsPerThread / 4];
	unsigned own = 0;
#pragma unroll
	for (int j = 0; j < kBinsPerThread / 4; j++) {
		v[j] = tv[j];
		own += v[j].x + v[j].y + v[j].z + v[j].w;
	}
	unsigned x = own;
	for (int o = 1; o < 32; o <<= 1) {
		const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
		if ((t & 31) >= o)
			x += y;
	}
	if ((t & 31) == 31)
		warp_sum[t >> 5] = x;
	__syncthreads();
	if (t < 32) {
		const unsigned w = warp_sum[t];
		unsigned z = w;
		for (int o = 1; o < 32; o <<= 1) {
			const unsigned y = __shfl_up_sync(0xffffffffu, z, o);
			if (t >= o)
				z += y;
		}
		warp_sum[t] = z - w;
	}
	__syncthreads();
	unsigned run = warp_sum[t >> 5] + x - own;
	uint4 *hv = reinterpret_cast<uint4 *>(h) + t * (kBinsPerThread / 4);
#pragma unroll
	for (int j = 0; j < kBinsPerThread / 4; j++) {
		uint4 o;
		o.x = run;
		o.y = o.x + v[j].x;
		o.z = o.y + v[j].y;
		o.w = o.z + v[j].z;
		run = o.w + v[j].w;
		hv[j] = o;
	}
}

// Measured on the 1.31M-triangle 1080p frame (sorts per frame): one pass 9.43 ms,
// two 8.46 ms, four 10.65 ms, eight 15.1 ms (every pass walks the whole chunk).
constexpr int kScatterPasses = 2;
static_assert(kBins % kScatterPasses == 0, "each scatter pass takes a whole range of bins");

// Block b's share of bin k starts at start[k] + hist[b][k], start being the exclusive
// scan of the bin totals (bins[0, kBins)), which every block computes for itself;
// block 0 also stores it in bins[kBins, 2 kBins) for the second-level sort.
__global__ void __launch_bounds__(1024) k_wf_bin_scatter(BinSrc src, unsigned *bins, const unsigned *hist,
                                                         int *status) {
	extern __shared__ __align__(16) unsigned h[];
	__shared__ unsigned warp_sum[kScanThreads / 32];
	block_scan_bins(bins, h, warp_sum);
	__syncthreads();
	{
		const uint4 *row = reinterpret_cast<const uint4 *>(hist + static_cast<size_t>(blockIdx.x) * kBins);
		uint4 *hv = reinterpret_cast<uint4 *>(h);
		uint4 *starts = reinterpret_cast<uint4 *>(bins + kBins);
		for (int b = threadIdx.x; b < kBins / 4; b += blockDim.x) {
			const uint4 r = row[b], o = hv[b];
			if (blockIdx.x == 0)
				starts[b] = o;
			hv[b] = make_uint4(o.x + r.x, o.y + r.y, o.z + r.z, o.w + r.w);
		}
	}
	__syncthreads();
	const unsigned n = *src.count;
	unsigned c0, c1;
	bin_chunk(n, blockIdx.x, gridDim.x, c0, c1);
	// kScatterPasses passes over the chunk, each placing the items of one range of
	// bins: fewer partly written output sectors are open at a time when the keys
	// arrive in random order (a later pass only re-reads the keys).
	for (int pass = 0; pass < kScatterPasses; pass++) {
		for (unsigned i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
			const unsigned key = src.keys[i] & (kBins - 1);
			if (static_cast<int>(key / (kBins / kScatterPasses)) != pass)
				continue;
			const unsigned pos = atomicAdd(&h[key], 1u);
			if (kBoundsCheck && pos >= n) {
				atomicOr(status, 1);
				continue;
			}
			src.out[pos] = src.items ? src.items[i] : static_cast<int>(i);
			if (src.fine)
				src.fine_out[pos] = src.fine[i];
		}
	}
}

// Second level of the ray sort: block b takes origin cell b's entries of the first
// level's output (starts holds the exclusive cell starts, so the cell spans
// [bins[b], bins[b+1]), the last one up to the item count) and places them by their
// 8-bit direction cell with a shared-memory counting sort. The queue ends up ordered by (origin cell,
// direction cell); entries of one bin keep no particular order.
constexpr int kFineBins = 256;
__global__ void __launch_bounds__(kFineBins) k_wf_bin_refine(const unsigned *starts, const unsigned *count,
                                                             const int *in, const uint8_t *fine, int *out,
                                                             unsigned n_max, int *status) {
	__shared__ unsigned h[kFineBins];
	__shared__ unsigned wsum[kFineBins / 32];
	const unsigned s = starts[blockIdx.x];
	const unsigned e = blockIdx.x + 1 < kBins ? starts[blockIdx.x + 1] : *count;
	if (e <= s) // the same for every thread of the block
		return;
	if (kBoundsCheck && e > n_max) {
		if (threadIdx.x == 0)
			atomicOr(status, 1);
		return;
	}
	const int t = threadIdx.x;
	h[t] = 0;
	__syncthreads();
	for (unsigned i = s + t; i < e; i += kFineBins)
		atomicAdd(&h[fine[i]], 1u);
	__syncthreads();
	// exclusive scan of the kFineBins counts, one per thread
	const unsigned c = h[t];
	unsigned x = c;
	for (int o = 1; o < 32; o <<= 1) {
		const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
		if ((t & 31) >= o)
			x += y;
	}
	if ((t & 31) == 31)
		wsum[t >> 5] = x;
	__syncthreads();
	if (t < 32) {
		const unsigned w = t < kFineBins / 32 ? wsum[t] : 0u;
		unsigned z = w;
		for (int o = 1; o < 32; o <<= 1) {
			const unsigned y = __shfl_up_sync(0xffffffffu, z, o);
			if (t >= o)
				z += y;
		}
		if (t < kFineBins / 32)
			wsum[t] = z - w;
	}
	__syncthreads();
	h[t] = s + wsum[t >> 5] + x - c;
	__syncthreads();
	for (unsigned i = s + t; i < e; i += kFineBins) {
		const unsigned pos = atomicAdd(&h[fine[i]], 1u);
		if (kBoundsCheck && pos >= e) {
			atomicOr(status, 1);
			continue;
		}
		out[pos] = in[i];
	}
}

// Three launches; `grid` <= kBinBlocksMax (the rows of hist). bins holds 2 kBins words.
cudaError_t bin_sort(const BinSrc &src, unsigned *bins, unsigned *hist, int grid, int *status, cudaStream_t st) {
	k_wf_bin_count<<<grid, 1024, kBins * sizeof(unsigned), st>>>(src, hist);
	k_wf_bin_colscan<<<kBins * kColSplit / kColScanThreads, kColScanThreads, 0, st>>>(hist, grid, bins);
	k_wf_bin_scatter<<<grid, 1024, kBins * sizeof(unsigned), st>>>(src, bins, hist, status);
	return cudaGetLastError();
}

// End of an adjoint wave: each path's radiance C is final, so every listed
// continuation vertex adds g (C - P) d log w / d albedo to its triangle.
__global__ void __launch_bounds__(256) k_wf_adj_flush(const WfJob *__restrict__ jobs, WfPool pool, WfWave wave) {
	__shared__ float agg[8 * 96];
	float *scratch = agg + (threadIdx.x >> 5) * 96;
	const int stride = gridDim.x * blockDim.x;
	// the loop bound is a multiple of the block size, so whole warps run each iteration
	const int end = (wave.n_slots + blockDim.x - 1) / blockDim.x * blockDim.x;
	for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < end; slot += stride) {
		const bool in = slot < wave.n_slots;
		const int n = in ? pool.adj_n[slot] : 0;
		F3 C = f3(0.0f, 0.0f, 0.0f), g = C;
		if (n > 0) {
			const float4 L = pool.L[slot];
			C = f3(L.x, L.y, L.z);
			g = adj_weight(jobs[__float_as_int(L.w)], pool.pixel[slot]);
		}
		const int n_warp = __reduce_max_sync(0xffffffffu, static_cast<unsigned>(n));
		for (int e = 0; e < n_warp; e++) {
			const bool on = e < n;
			int tri = 0;
			F3 v = f3(0.0f, 0.0f, 0.0f);
			if (on) {
				const size_t at = static_cast<size_t>(e) * pool.capacity + slot;
				const float4 P = pool.adj_pt[at], dl = pool.adj_dlog[at];
				tri = __float_as_int(dl.w);
				v = g * (C - f3(P.x, P.y, P.z)) * f3(dl.x, dl.y, dl.z);
			}
			add_grad3_warp(pool.d_alb, tri, v, on, 0xffffffffu, scratch);
		}
	}
}

// Adds each pixel's samples of this wave to its sum, in sample order.
__global__ void __launch_bounds__(256) k_wf_accumulate(const WfJob *__restrict__ jobs, WfPool pool, WfWave wave) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < wave.n_pix; i += gridDim.x * blockDim.x) {
		const int a = find_base(wave.pbases, wave.n_jobs, i);
		const WfJob &job = jobs[wave.jobs[a]];
		const int pixel = i - wave.pbases[a];
		const int base = wave.bases[a] + pixel;
		float *acc = job.accum + 3 * static_cast<size_t>(pixel);
		float sx = acc[0], sy = acc[1], sz = acc[2];
		for (int k = 0; k < wave.nsamp[a]; k++) {
			const float4 L = pool.L[base + k * job.n_pix];
			sx = sx + L.x;
			sy = sy + L.y;
			sz = sz + L.z;
		}
		acc[0] = sx;
		acc[1] = sy;
		acc[2] = sz;
	}
}

} // namespace

cudaError_t wf_launch_wave(const WfJob *d_jobs, const WfPool &pool, const WfWave &wave, int max_depth, int order,
                           const WfLaunch &lc, int *status, cudaStream_t st) {
	if (wave.n_slots <= 0)
		return cudaSuccess;
	cudaError_t e = cudaMemsetAsync(pool.counters, 0, kCntTotal * sizeof(unsigned), st);
	if (e != cudaSuccess)
		return e;
	// adjoint waves: every slot's continuation list starts empty; their traversal stages
	// are the one-ray-per-lane kernels, whose shadow stage adds the next-event terms
	const bool adj = pool.adj_n != nullptr;
	if (adj) {
		e = cudaMemsetAsync(pool.adj_n, 0, static_cast<size_t>(wave.n_slots) * sizeof(int), st);
		if (e != cudaSuccess)
			return e;
	}
	// profiled frames: an event after every stage (no effect on the work)
	auto mark = [&](int stage, int kernels) -> cudaError_t {
		return lc.clock ? lc.clock->mark(stage, kernels, st) : cudaSuccess;
	};
	const int gcam = (wave.n_slots + 255) / 256 < 148 * 8 ? (wave.n_slots + 255) / 256 : 148 * 8;
	k_wf_camera<<<gcam, 256, 0, st>>>(d_jobs, pool, wave);
	if ((e = mark(kStCamera, 1)) != cudaSuccess)
		return e;
	const bool use_dyn = lc.dyn && order == kOrderReference && !adj;
	const bool sort = lc.sort && pool.keys && pool.fine && pool.sorted_coarse && pool.sorted_fine && pool.sorted &&
	                  pool.bins && pool.bin_hist && lc.grid_bin >= 1 && lc.grid_bin <= kBinBlocksMax;
	for (int k = 0; k < max_depth; k++) {
		const int *q = pool.queue[k & 1];
		if (sort && k > 0) {
			e = bin_sort(BinSrc{pool.keys, pool.counters + kCntRays + k, q, pool.sorted_coarse, pool.fine,
			                    pool.sorted_fine},
			             pool.bins, pool.bin_hist, lc.grid_bin, status, st);
			if (e != cudaSuccess)
				return e;
			k_wf_bin_refine<<<kBins, kFineBins, 0, st>>>(pool.bins + kBins, pool.counters + kCntRays + k, pool.sorted_coarse,
			                                            pool.sorted_fine, pool.sorted,
			                                            static_cast<unsigned>(pool.capacity), status);
			q = pool.sorted;
			if ((e = mark(kStRaySort, 4)) != cudaSuccess)
				return e;
		}
		const int oj = wave.only_job;
		if (use_dyn)
			k_wf_trace_dyn<false><<<lc.grid_dyn, 128, 0, st>>>(d_jobs, pool, k, q, oj, status);
		else if (order == kOrderNearest)
			k_wf_extend<kOrderNearest><<<lc.grid_ext, 128, kWfExtendSmem, st>>>(d_jobs, pool, k, q, oj, status);
		else
			k_wf_extend<kOrderReference><<<lc.grid_ext, 128, kWfExtendSmem, st>>>(d_jobs, pool, k, q, oj, status);
		if ((e = mark(kStExtend, 1)) != cudaSuccess)
			return e;
		// Shading takes the queue in its append order, not the binned order: the previous
		// bounce appended each warp's surviving slots in increasing order, so the path
		// state reads and writes of neighbouring lanes fall on neighbouring slots. The
		// first bounce shades every slot in slot order (its queue is in pixel-tile order
		// for the closest-hit stage). The results do not depend on the order in which
		// paths are shaded.
		const int *qs = k == 0 ? nullptr : pool.queue[k & 1];
		if (adj)
			k_wf_shade<true><<<lc.grid_shade, 128, 0, st>>>(d_jobs, pool, k, qs, sort ? 1 : 0, status);
		else
			k_wf_shade<false><<<lc.grid_shade, 128, 0, st>>>(d_jobs, pool, k, qs, sort ? 1 : 0, status);
		if ((e = mark(kStShade, 1)) != cudaSuccess)
			return e;
		if (use_dyn)
			k_wf_trace_dyn<true><<<lc.grid_dyn, 128, 0, st>>>(d_jobs, pool, k, nullptr, oj, status);
		else {
			// with binning, the shadow records are traced in the order of their origins' cells
			// and sub-cells; the ray sort's first-level buffers are free until the next bounce
			const bool sort_sh = sort && pool.sh_keys && pool.sh_fine && pool.sh_sorted;
			if (sort_sh) {
				e = bin_sort(BinSrc{pool.sh_keys, pool.counters + kCntShadow + k, nullptr, pool.sorted_coarse,
				                    pool.sh_fine, pool.sorted_fine},
				             pool.bins, pool.bin_hist, lc.grid_bin, status, st);
				if (e != cudaSuccess)
					return e;
				k_wf_bin_refine<<<kBins, kFineBins, 0, st>>>(pool.bins + kBins, pool.counters + kCntShadow + k,
				                                            pool.sorted_coarse, pool.sorted_fine, pool.sh_sorted,
				                                            static_cast<unsigned>(pool.capacity), status);
				if ((e = mark(kStShadowSort, 4)) != cudaSuccess)
					return e;
			}
			const int *order_sh = sort_sh ? pool.sh_sorted : nullptr;
			if (adj)
				k_wf_shadow<true><<<lc.grid_sh, 128, kWfShadowSmem, st>>>(d_jobs, pool, k, oj, order_sh, status);
			else
				k_wf_shadow<false><<<lc.grid_sh, 128, kWfShadowSmem, st>>>(d_jobs, pool, k, oj, order_sh, status);
		}
		if ((e = mark(kStShadow, 1)) != cudaSuccess)
			return e;
	}
	if (adj) {
		k_wf_adj_flush<<<gcam, 256, 0, st>>>(d_jobs, pool, wave);
		return cudaGetLastError();
	}
	const int gacc = (wave.n_pix + 255) / 256 < 148 * 8 ? (wave.n_pix + 255) / 256 : 148 * 8;
	k_wf_accumulate<<<gacc, 256, 0, st>>>(d_jobs, pool, wave);
	if ((e = mark(kStAccumulate, 1)) != cudaSuccess)
		return e;
	return cudaGetLastError();
}

// Persistent grid sizes (blocks resident on all SMs).
void wf_grid_sizes(int &grid_ext, int &grid_shade, int &grid_sh, int &grid_dyn, int &grid_bin) {
	int dev = 0, sms = 148;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	int a = 0, b = 0, c = 0, d0 = 0, d1 = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_wf_extend<kOrderReference>, 128, kWfExtendSmem);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_wf_shade<false>, 128, 0);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, k_wf_shadow<false>, 128, kWfShadowSmem);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d0, k_wf_trace_dyn<false>, 128, 0);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d1, k_wf_trace_dyn<true>, 128, 0);
	grid_ext = sms * (a > 0 ? a : 1);
	grid_shade = sms * (b > 0 ? b : 1);
	grid_sh = sms * (c > 0 ? c : 1);
	const int d = d0 < d1 ? d0 : d1;
	grid_dyn = sms * (d > 0 ? d : 1);
	grid_bin = sms < kBinBlocksMax ? sms : kBinBlocksMax; // one 1024-thread block per SM
	constexpr int kHist = kBins * static_cast<int>(sizeof(unsigned));
	if (kHist > 48 * 1024) {
		cudaFuncSetAttribute(k_wf_bin_count, cudaFuncAttributeMaxDynamicSharedMemorySize, kHist);
		cudaFuncSetAttribute(k_wf_bin_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, kHist);
	}
}

} // namespace rnb
