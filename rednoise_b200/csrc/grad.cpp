// Differentiable-rendering entry points: material updates and the adjoint.
#include <algorithm>
#include <cstring>
#include <vector>

#include "adjoint.hpp"
#include "render_impl.hpp"
#include "scene_impl.hpp"
#include "trace_range.hpp"
#include "wavefront_host.hpp"

using namespace rnb;

namespace {

// The adjoint as wavefront waves (one job per view): the paths are regenerated and
// traced once, in waves sorted like rn_pt_render's wavefront, each path keeping its
// continuation vertices in the pool until its radiance is final.
rn_status backward_wavefront(rn_scene *scene, const PhysScene &ps, const std::vector<AdjView> &views, float *g_alb,
                             float *g_em, cudaStream_t cs) {
	std::vector<WfJob> jobs(views.size());
	int max_depth = 1, max_spp = 0;
	long pix = 0;
	for (size_t v = 0; v < views.size(); v++) {
		WfJob &j = jobs[v];
		j.sc = ps;
		j.cam = views[v].cam;
		j.st = views[v].st;
		j.accum = nullptr;
		j.n_pix = views[v].n_pix;
		j.spp = views[v].st.spp > 0 ? views[v].st.spp : 0;
		j.dimg = views[v].dimg;
		max_depth = std::max(max_depth, j.st.max_depth);
		max_spp = std::max(max_spp, j.spp);
		if (j.spp > 0)
			pix += j.n_pix;
	}
	if (max_spp == 0 || pix == 0)
		return RN_OK;
	const int entries = std::max(1, max_depth - 1);
	size_t budget = 0;
	RNB_CUDA(wf_pool_budget(budget));
	long spw = static_cast<long>(budget / (wf_adjoint_bytes_per_path(entries) * static_cast<size_t>(pix)));
	spw = std::min<long>(spw, (1L << 30) / pix);
	spw = std::max<long>(1, std::min<long>(spw, max_spp));
	if (!scene->wf_adj)
		scene->wf_adj.reset(new WfContext());
	WfContext &wf = *scene->wf_adj;
	wf.set_frame_io(nullptr, 0, {});
	wf.set_dynamic(0);
	wf.set_sort(1);
	wf.set_adjoint(entries, g_alb, g_em);
	rn_status r = wf.configure(jobs, max_depth, kOrderReference, static_cast<int>(spw), cs);
	if (r != RN_OK)
		return r;
	return wf.enqueue(scene->d_status.as<int>(), cs);
}

} // namespace

extern "C" {

rn_status rn_pt_scene_set_materials(rn_scene *scene, const float *albedo, const float *emission, unsigned flags,
                                    void *stream) {
	if (!scene) {
		set_last_error("rn_pt_scene_set_materials: NULL scene");
		return RN_ERR_INVALID_ARGUMENT;
	}
	rn_status r = prepare_scene(scene);
	if (r != RN_OK)
		return r;
	const int n = static_cast<int>(scene->tris.size());
	cudaStream_t cs = pick_stream(scene, stream);
	if (flags & RN_PT_DEVICE_POINTERS)
		return launch_set_materials(scene->d_phys_shade.as<float4>(), n, albedo, emission, cs) == cudaSuccess
		           ? RN_OK
		           : cuda_fail(cudaGetLastError(), "launch_set_materials");
	// Host arrays: keep the host copies in step and stage the upload.
	const size_t bytes = static_cast<size_t>(n) * 3 * sizeof(float);
	std::lock_guard<std::mutex> lock(scene->scratch_mu);
	RNB_CUDA(scene->scratch.ensure(2 * bytes + 256));
	float *d_a = albedo ? scene->scratch.as<float>() : nullptr;
	float *d_e = emission ? scene->scratch.as<float>() + 3 * static_cast<size_t>(n) + 64 : nullptr;
	if (albedo) {
		std::memcpy(scene->tris.albedo.data(), albedo, bytes);
		RNB_CUDA(cudaMemcpyAsync(d_a, albedo, bytes, cudaMemcpyHostToDevice, cs));
	}
	if (emission) {
		RNB_CUDA(cudaMemcpyAsync(d_e, emission, bytes, cudaMemcpyHostToDevice, cs));
	}
	RNB_CUDA(launch_set_materials(scene->d_phys_shade.as<float4>(), n, d_a, d_e, cs));
	RNB_CUDA(cudaStreamSynchronize(cs));
	return RN_OK;
}

rn_status rn_pt_backward(rn_scene *scene, int n_views, const rn_pt_camera *cameras, const rn_pt_settings *settings,
                         const float *const *d_images, unsigned flags, void *stream, float *d_albedo,
                         float *d_emission) {
	TraceRange trace_range("rn_pt_backward");
	if (!scene || n_views <= 0 || !cameras || !settings || !d_images) {
		set_last_error("rn_pt_backward: invalid argument");
		return RN_ERR_INVALID_ARGUMENT;
	}
	std::vector<AdjView> views(static_cast<size_t>(n_views));
	std::vector<long> pix_base(static_cast<size_t>(n_views));
	PhysScene ps{};
	long total = 0, items = 0;
	for (int v = 0; v < n_views; v++) {
		PhysCamera pc;
		PhysSettings pst;
		rn_status r = make_phys_inputs(scene, &cameras[v], &settings[v], 0, ps, pc, pst);
		if (r != RN_OK)
			return r;
		if (!d_images[v]) {
			set_last_error("rn_pt_backward: NULL image gradient");
			return RN_ERR_INVALID_ARGUMENT;
		}
		views[v].cam = pc;
		views[v].st = pst;
		views[v].n_pix = pc.width * pc.height;
		views[v].item_base = static_cast<unsigned>(items);
		pix_base[v] = total;
		total += views[v].n_pix;
		items += static_cast<long>(views[v].n_pix) * (pst.spp > 0 ? pst.spp : 0);
		if (total > (1L << 30) || items > (1L << 31)) {
			set_last_error("rn_pt_backward: more than 2^30 pixels or 2^31 (pixel, sample) pairs");
			return RN_ERR_CAPACITY;
		}
	}
	const int n = static_cast<int>(scene->tris.size());
	const bool dev = (flags & RN_PT_DEVICE_POINTERS) != 0;
	cudaStream_t cs = pick_stream(scene, stream);
	const size_t gbytes = static_cast<size_t>(n) * 3 * sizeof(float);
	std::unique_lock<std::mutex> lock(scene->scratch_mu);
	// Scratch: view table, gradient buffers, and (host mode) the image gradients.
	const size_t vbytes = (views.size() * sizeof(AdjView) + 255) & ~size_t(255);
	const size_t gb = (gbytes + 255) & ~size_t(255);
	const size_t ib = dev ? 0 : static_cast<size_t>(total) * 3 * sizeof(float);
	// Device mode returns without a host synchronisation, so its view table lives in
	// a buffer of its own (calls on one scene are ordered on the caller's stream).
	DevBuf &buf = dev ? scene->adj : scene->scratch;
	RNB_CUDA(buf.ensure(vbytes + 2 * gb + ib + 256));
	char *base = buf.as<char>();
	AdjView *d_views = reinterpret_cast<AdjView *>(base);
	float *g_alb = (dev && d_albedo) ? d_albedo : reinterpret_cast<float *>(base + vbytes);
	float *g_em = (dev && d_emission) ? d_emission : reinterpret_cast<float *>(base + vbytes + gb);
	float *imgs = reinterpret_cast<float *>(base + vbytes + 2 * gb);
	for (int v = 0; v < n_views; v++) {
		if (dev) {
			views[v].dimg = d_images[v];
		} else {
			float *dst = imgs + 3 * static_cast<size_t>(pix_base[v]);
			RNB_CUDA(cudaMemcpyAsync(dst, d_images[v], static_cast<size_t>(views[v].n_pix) * 12,
			                         cudaMemcpyHostToDevice, cs));
			views[v].dimg = dst;
		}
	}
	RNB_CUDA(cudaMemcpyAsync(d_views, views.data(), views.size() * sizeof(AdjView), cudaMemcpyHostToDevice, cs));
	RNB_CUDA(cudaMemsetAsync(g_alb, 0, gbytes, cs));
	RNB_CUDA(cudaMemsetAsync(g_em, 0, gbytes, cs));
	// Integrator: RN_PT_MEGAKERNEL in any view's settings keeps one thread per path,
	// RN_PT_WAVEFRONT in any view asks for waves; RN_PT_AUTO takes waves above the
	// triangle count whose gradients the per-path kernel keeps in shared memory.
	bool want_mk = false, want_wf = false, depth_ok = true;
	for (int v = 0; v < n_views; v++) {
		want_mk = want_mk || settings[v].integrator == RN_PT_MEGAKERNEL;
		want_wf = want_wf || settings[v].integrator == RN_PT_WAVEFRONT;
		depth_ok = depth_ok && views[v].st.max_depth <= kWfMaxDepth;
	}
	const bool use_wf = depth_ok && !want_mk && (want_wf || n > kAdjointSharedTris);
	if (use_wf) {
		rn_status r = backward_wavefront(scene, ps, views, g_alb, g_em, cs);
		if (r != RN_OK)
			return r;
	} else {
		RNB_CUDA(scene->d_adj_counter.ensure(256));
		RNB_CUDA(launch_adjoint(ps, d_views, n_views, static_cast<unsigned>(items), g_alb, g_em, n,
		                        scene->d_adj_counter.as<unsigned>(), scene->d_status.as<int>(), cs));
	}
	if (dev)
		return RN_OK;
	if (d_albedo)
		RNB_CUDA(cudaMemcpyAsync(d_albedo, g_alb, gbytes, cudaMemcpyDeviceToHost, cs));
	if (d_emission)
		RNB_CUDA(cudaMemcpyAsync(d_emission, g_em, gbytes, cudaMemcpyDeviceToHost, cs));
	int h = 0;
	RNB_CUDA(cudaMemcpyAsync(&h, scene->d_status.p, sizeof(int), cudaMemcpyDeviceToHost, cs));
	RNB_CUDA(cudaStreamSynchronize(cs));
	if (h) {
		set_last_error("rn_pt_backward: device status word reports a traversal error");
		return RN_ERR_INTERNAL;
	}
	return RN_OK;
}

} // extern "C"
