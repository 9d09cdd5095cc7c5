// Physical-mode rendering entry points (rn_pt_render / rn_pt_render_accumulate).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "pt_kernels.hpp"
#include "render_impl.hpp"
#include "scene_impl.hpp"
#include "trace_range.hpp"

namespace rnb {

rn_status make_phys_inputs(rn_scene *s, const rn_pt_camera *c, const rn_pt_settings *st, unsigned flags,
                           PhysScene &ps, PhysCamera &pc, PhysSettings &pst) {
	if (!s || !c || !st) {
		set_last_error("render: NULL argument");
		return RN_ERR_INVALID_ARGUMENT;
	}
	if (c->width <= 0 || c->height <= 0 || static_cast<long>(c->width) * c->height > (1L << 28)) {
		set_last_error("render: camera width/height must be positive and at most 2^28 pixels");
		return RN_ERR_INVALID_ARGUMENT;
	}
	if (!(c->vfov_deg > 0.0f && c->vfov_deg < 179.0f)) {
		set_last_error("render: vfov_deg must be in (0, 179)");
		return RN_ERR_INVALID_ARGUMENT;
	}
	if (st->spp < 0 || st->max_depth < 1 || st->max_depth > 64) {
		set_last_error("render: need spp >= 0 and 1 <= max_depth <= 64");
		return RN_ERR_INVALID_ARGUMENT;
	}
	rn_status r = prepare_scene(s);
	if (r != RN_OK)
		return r;
	ps.sv = s->view;
	ps.shade = s->d_phys_shade.as<float4>();
	ps.emitters = s->d_emitters.as<float4>();
	ps.n_emitters = s->n_emitters;
	ps.emit_area_total = s->emit_area_total;

	double pos[3], fwd[3], up[3], right[3], upv[3];
	for (int a = 0; a < 3; a++) {
		pos[a] = c->position[a];
		fwd[a] = static_cast<double>(c->target[a]) - c->position[a];
		up[a] = c->up[a];
	}
	auto nrm = [](double v[3]) {
		const double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
		if (l > 0)
			for (int a = 0; a < 3; a++)
				v[a] /= l;
		return l > 0;
	};
	auto crs = [](const double a[3], const double b[3], double o[3]) {
		o[0] = a[1] * b[2] - a[2] * b[1];
		o[1] = a[2] * b[0] - a[0] * b[2];
		o[2] = a[0] * b[1] - a[1] * b[0];
	};
	if (!nrm(fwd)) {
		set_last_error("render: camera target equals its position");
		return RN_ERR_INVALID_ARGUMENT;
	}
	crs(fwd, up, right);
	if (!nrm(right)) {
		set_last_error("render: camera up is parallel to the view direction");
		return RN_ERR_INVALID_ARGUMENT;
	}
	crs(right, fwd, upv);
	for (int a = 0; a < 3; a++) {
		pc.pos[a] = static_cast<float>(pos[a]);
		pc.fwd[a] = static_cast<float>(fwd[a]);
		pc.right[a] = static_cast<float>(right[a]);
		pc.up[a] = static_cast<float>(upv[a]);
	}
	pc.tan_half_y = static_cast<float>(std::tan(c->vfov_deg * 3.14159265358979323846 / 360.0));
	pc.aspect = static_cast<float>(c->width) / static_cast<float>(c->height);
	pc.width = c->width;
	pc.height = c->height;
	pst.spp = st->spp;
	pst.max_depth = st->max_depth;
	pst.rr_depth = st->rr_depth;
	pst.order = (flags & RN_PT_ORDER_NEAREST) ? kOrderNearest : kOrderReference;
	if (flags & RN_PT_LBVH) { // the GPU-built tree, nearest child first
		if (!s->lbvh_ready) {
			set_last_error("render: RN_PT_LBVH needs rn_pt_scene_build_lbvh first");
			return RN_ERR_INVALID_ARGUMENT;
		}
		ps.sv = s->lbvh_view;
		pst.order = kOrderNearest;
	}
	pst.seed = st->seed;
	pst.sample_offset = st->sample_offset;
	for (int a = 0; a < 3; a++)
		pst.env[a] = st->env[a];
	return RN_OK;
}

} // namespace rnb

using namespace rnb;

namespace {

// Run one integrator over accum (device, 3 floats per pixel). spw <= 0 picks the
// default samples per wave; dyn selects the wavefront's per-lane ray replacement
// and sort its binning of each bounce's rays.
rn_status run_fixed(rn_scene *s, int integrator, int spw, int dyn, int sort, const PhysScene &ps,
                    const PhysCamera &pc, const PhysSettings &pst, float *d_accum, cudaStream_t cs,
                    WfStageClock *clock = nullptr) {
	if (integrator == RN_PT_WAVEFRONT) {
		if (pst.max_depth > kWfMaxDepth) {
			set_last_error("render: the wavefront integrator supports max_depth <= 64");
			return RN_ERR_INVALID_ARGUMENT;
		}
		if (!s->wf)
			s->wf.reset(new WfContext());
		WfJob job;
		job.sc = ps;
		job.cam = pc;
		job.st = pst;
		job.accum = d_accum;
		job.n_pix = pc.width * pc.height;
		job.spp = pst.spp;
		s->wf->set_frame_io(nullptr, 0, {});
		s->wf->set_dynamic(dyn);
		s->wf->set_sort(sort);
		if (spw <= 0)
			spw = default_samples_per_wave(job.n_pix, job.spp);
		rn_status r = s->wf->configure({job}, pst.max_depth, pst.order, spw, cs);
		if (r != RN_OK)
			return r;
		if (clock) // profiled frame: the same launches, made directly with stage events
			return s->wf->enqueue(s->d_status.as<int>(), cs, clock);
		return s->wf->launch_graph(s->d_status.as<int>(), cs);
	}
	RNB_CUDA(s->d_counter.ensure(256));
	RNB_CUDA(launch_megakernel(ps, pc, pst, d_accum, s->d_counter.as<unsigned>(), s->d_status.as<int>(), cs));
	return RN_OK;
}

std::tuple<int, int, int, int> tune_key(const PhysCamera &pc, const PhysSettings &pst) {
	return {pc.width, pc.height, pst.max_depth, pst.order};
}

// Measure the candidates on up to 64 samples per pixel and remember the fastest:
// the megakernel, and the wavefront with and without binning each bounce's rays
// and with and without per-lane ray replacement in its traversal stages (at the
// largest queue capacity), then the queue capacity itself, from the default up to
// a whole frame's paths in one wave, within a memory budget.
rn_status autotune_scene(rn_scene *s, const PhysScene &ps, const PhysCamera &pc, const PhysSettings &pst,
                         rn_pt_tuning &out) {
	TraceRange trace_range("autotune");
	PhysSettings probe = pst;
	probe.spp = std::clamp(pst.spp, 1, 64);
	probe.sample_offset = 0x40000000u;
	const long n_pix = static_cast<long>(pc.width) * pc.height;
	const size_t bytes = static_cast<size_t>(n_pix) * 3 * sizeof(float);
	RNB_CUDA(s->tune_accum.ensure(bytes));
	float *acc = s->tune_accum.as<float>();
	cudaStream_t cs = s->stream;
	struct Events {
		cudaEvent_t a = nullptr, b = nullptr;
		~Events() {
			if (a)
				cudaEventDestroy(a);
			if (b)
				cudaEventDestroy(b);
		}
	} ev;
	RNB_CUDA(cudaEventCreate(&ev.a));
	RNB_CUDA(cudaEventCreate(&ev.b));
	const double samples = static_cast<double>(n_pix) * probe.spp;
	auto time_one = [&](int integ, int spw, int dyn, int sort, double &sps) -> rn_status {
		for (int rep = 0; rep < 2; rep++) { // the first run warms caches and captures graphs
			RNB_CUDA(cudaMemsetAsync(acc, 0, bytes, cs));
			RNB_CUDA(cudaEventRecord(ev.a, cs));
			rn_status r = run_fixed(s, integ, spw, dyn, sort, ps, pc, probe, acc, cs);
			if (r != RN_OK)
				return r;
			RNB_CUDA(cudaEventRecord(ev.b, cs));
		}
		RNB_CUDA(cudaEventSynchronize(ev.b));
		float ms = 0.0f;
		RNB_CUDA(cudaEventElapsedTime(&ms, ev.a, ev.b));
		sps = ms > 0.0f ? samples / (ms * 1e-3) : 0.0;
		return RN_OK;
	};
	rn_status r = time_one(RN_PT_MEGAKERNEL, 0, 0, 0, out.megakernel_sps);
	if (r != RN_OK)
		return r;
	// Queue capacities: d, 2d, 4d, ... samples per wave, at most the probe's spp, with
	// the path pool within half the free memory and 32 GiB.
	size_t budget = 0;
	RNB_CUDA(wf_pool_budget(budget));
	std::vector<int> spws;
	for (int k = default_samples_per_wave(n_pix, probe.spp); k <= probe.spp; k *= 2) {
		if (!spws.empty() && static_cast<size_t>(n_pix) * k * kWfBytesPerPath > budget)
			break;
		spws.push_back(k);
	}
	const int widest = spws.back();
	out.wavefront_sps = 0.0;
	out.samples_per_wave = widest;
	out.dynamic_fetch = 0;
	out.ray_sort = 0;
	for (int sort : {0, 1}) {
		for (int dyn : {0, 1}) {
			if (dyn && pst.order != kOrderReference)
				continue;
			double sps = 0.0;
			r = time_one(RN_PT_WAVEFRONT, widest, dyn, sort, sps);
			if (r != RN_OK)
				return r;
			if (sps > out.wavefront_sps) {
				out.wavefront_sps = sps;
				out.dynamic_fetch = dyn;
				out.ray_sort = sort;
			}
		}
	}
	for (int spw : spws) {
		if (spw == widest)
			continue;
		double sps = 0.0;
		r = time_one(RN_PT_WAVEFRONT, spw, out.dynamic_fetch, out.ray_sort, sps);
		if (r != RN_OK)
			return r;
		if (sps > out.wavefront_sps) {
			out.wavefront_sps = sps;
			out.samples_per_wave = spw;
		}
	}
	out.integrator = out.wavefront_sps > out.megakernel_sps ? RN_PT_WAVEFRONT : RN_PT_MEGAKERNEL;
	s->tuned[tune_key(pc, pst)] = {out.integrator, out.samples_per_wave, out.dynamic_fetch, out.ray_sort};
	return RN_OK;
}

// Run the integrator the settings ask for; RN_PT_AUTO uses (and on first use
// measures) the scene's tuned choice for this image size.
rn_status run_integrator(rn_scene *s, const rn_pt_settings *st, unsigned flags, const PhysScene &ps,
                         const PhysCamera &pc, const PhysSettings &pst, float *d_accum, cudaStream_t cs) {
	auto it = s->tuned.find(tune_key(pc, pst));
	// Ray binning: forced on or off by the flags, else the tuned choice.
	auto pick_sort = [flags](int tuned) {
		return (flags & RN_PT_RAY_SORT) ? 1 : ((flags & RN_PT_NO_RAY_SORT) ? 0 : tuned);
	};
	if (st->integrator == RN_PT_MEGAKERNEL)
		return run_fixed(s, RN_PT_MEGAKERNEL, 0, 0, 0, ps, pc, pst, d_accum, cs);
	if (st->integrator == RN_PT_WAVEFRONT) {
		// An explicit wavefront render keeps the tuned wavefront choices when there are some.
		const int dyn = (flags & RN_PT_WAVEFRONT_STATIC) ? 0 : 1;
		if (it != s->tuned.end() && std::get<0>(it->second) == RN_PT_WAVEFRONT)
			return run_fixed(s, RN_PT_WAVEFRONT, std::get<1>(it->second), dyn ? std::get<2>(it->second) : 0,
			                 pick_sort(std::get<3>(it->second)), ps, pc, pst, d_accum, cs);
		return run_fixed(s, RN_PT_WAVEFRONT, 0, dyn, pick_sort(0), ps, pc, pst, d_accum, cs);
	}
	if (it == s->tuned.end()) {
		rn_pt_tuning t{};
		rn_status r = autotune_scene(s, ps, pc, pst, t);
		if (r != RN_OK)
			return r;
		it = s->tuned.find(tune_key(pc, pst));
	}
	const auto [integ, spw, dyn, sort] = it->second;
	return run_fixed(s, integ, spw, dyn, pick_sort(sort), ps, pc, pst, d_accum, cs);
}

// The wavefront configuration an RN_PT_AUTO render would use when its tuned choice
// is the wavefront, else the explicit wavefront's: (samples per wave, dyn, sort).
std::tuple<int, int, int> wavefront_choice(rn_scene *s, unsigned flags, const PhysCamera &pc,
                                           const PhysSettings &pst) {
	auto pick_sort = [flags](int tuned) {
		return (flags & RN_PT_RAY_SORT) ? 1 : ((flags & RN_PT_NO_RAY_SORT) ? 0 : tuned);
	};
	const bool static_lanes = (flags & RN_PT_WAVEFRONT_STATIC) != 0;
	auto it = s->tuned.find(tune_key(pc, pst));
	if (it != s->tuned.end() && std::get<0>(it->second) == RN_PT_WAVEFRONT)
		return {std::get<1>(it->second), static_lanes ? 0 : std::get<2>(it->second),
		        pick_sort(std::get<3>(it->second))};
	return {0, static_lanes ? 0 : 1, pick_sort(0)};
}

rn_status finish_sync(rn_scene *s, cudaStream_t cs, const char *what) {
	int h = 0;
	RNB_CUDA(cudaMemcpyAsync(&h, s->d_status.p, sizeof(int), cudaMemcpyDeviceToHost, cs));
	RNB_CUDA(cudaStreamSynchronize(cs));
	if (h) {
		cudaMemsetAsync(s->d_status.p, 0, sizeof(int), cs);
		set_last_error(std::string(what) + ": device status word reports a traversal error");
		return RN_ERR_INTERNAL;
	}
	return RN_OK;
}

} // namespace

extern "C" {

rn_status rn_pt_profile_wavefront(rn_scene *scene, const rn_pt_camera *camera, const rn_pt_settings *settings,
                                  unsigned flags, void *stream, float *rgb, rn_pt_stage_times *out) {
	TraceRange trace_range("rn_pt_profile_wavefront");
	PhysScene ps;
	PhysCamera pc;
	PhysSettings pst;
	rn_status r = make_phys_inputs(scene, camera, settings, flags, ps, pc, pst);
	if (r != RN_OK)
		return r;
	if (!rgb || !out) {
		set_last_error("rn_pt_profile_wavefront: NULL rgb or out");
		return RN_ERR_INVALID_ARGUMENT;
	}
	cudaStream_t cs = pick_stream(scene, stream);
	const long nf = static_cast<long>(camera->width) * camera->height * 3;
	const size_t bytes = static_cast<size_t>(nf) * sizeof(float);
	const float inv = settings->spp > 0 ? 1.0f / static_cast<float>(settings->spp) : 0.0f;
	std::lock_guard<std::mutex> lock(scene->scratch_mu);
	RNB_CUDA(scene->scratch.ensure(2 * bytes + 256));
	float *acc = scene->scratch.as<float>();
	float *mean = (flags & RN_PT_DEVICE_POINTERS) ? rgb : acc + nf + 64;
	const auto [spw, dyn, sort] = wavefront_choice(scene, flags, pc, pst);
	std::unique_ptr<WfStageClock> clock(new WfStageClock());
	RNB_CUDA(cudaMemsetAsync(acc, 0, bytes, cs));
	r = run_fixed(scene, RN_PT_WAVEFRONT, spw, dyn, sort, ps, pc, pst, acc, cs, clock.get());
	if (r != RN_OK)
		return r;
	RNB_CUDA(launch_resolve(acc, mean, nf, inv, cs));
	RNB_CUDA(clock->mark(kStAccumulate, 1, cs));
	if (!(flags & RN_PT_DEVICE_POINTERS))
		RNB_CUDA(cudaMemcpyAsync(rgb, mean, bytes, cudaMemcpyDeviceToHost, cs));
	r = finish_sync(scene, cs, "rn_pt_profile_wavefront");
	if (r != RN_OK)
		return r;
	if (clock->overflow) {
		set_last_error("rn_pt_profile_wavefront: more stages than the profiler records");
		return RN_ERR_CAPACITY;
	}
	double ms[kStCount] = {};
	cudaEvent_t prev = clock->start;
	for (int i = 0; i < clock->n; i++) {
		float t = 0.0f;
		RNB_CUDA(cudaEventElapsedTime(&t, prev, clock->ev[i]));
		ms[clock->kind[i]] += t;
		prev = clock->ev[i];
	}
	float total = 0.0f;
	if (clock->n > 0)
		RNB_CUDA(cudaEventElapsedTime(&total, clock->start, clock->ev[clock->n - 1]));
	out->camera_ms = ms[kStCamera];
	out->ray_sort_ms = ms[kStRaySort];
	out->extend_ms = ms[kStExtend];
	out->shade_ms = ms[kStShade];
	out->shadow_sort_ms = ms[kStShadowSort];
	out->shadow_ms = ms[kStShadow];
	out->accumulate_ms = ms[kStAccumulate];
	out->total_ms = total;
	out->launches = clock->launches;
	const int used_spw = spw > 0 ? spw : default_samples_per_wave(pc.width * static_cast<long>(pc.height), pst.spp);
	out->waves = pst.spp > 0 ? (pst.spp + used_spw - 1) / used_spw : 0;
	out->samples_per_wave = used_spw;
	out->dynamic_fetch = dyn;
	out->ray_sort = sort;
	return RN_OK;
}

rn_status rn_pt_render_accumulate(rn_scene *scene, const rn_pt_camera *camera, const rn_pt_settings *settings,
                                  unsigned flags, void *stream, float *accum) {
	TraceRange trace_range("rn_pt_render_accumulate");
	PhysScene ps;
	PhysCamera pc;
	PhysSettings pst;
	rn_status r = make_phys_inputs(scene, camera, settings, flags, ps, pc, pst);
	if (r != RN_OK)
		return r;
	if (!accum) {
		set_last_error("rn_pt_render_accumulate: NULL accum");
		return RN_ERR_INVALID_ARGUMENT;
	}
	cudaStream_t cs = pick_stream(scene, stream);
	const size_t bytes = static_cast<size_t>(camera->width) * camera->height * 3 * sizeof(float);
	if (flags & RN_PT_DEVICE_POINTERS)
		return run_integrator(scene, settings, flags, ps, pc, pst, accum, cs);
	std::lock_guard<std::mutex> lock(scene->scratch_mu);
	RNB_CUDA(scene->scratch.ensure(bytes));
	float *d = scene->scratch.as<float>();
	RNB_CUDA(cudaMemcpyAsync(d, accum, bytes, cudaMemcpyHostToDevice, cs));
	r = run_integrator(scene, settings, flags, ps, pc, pst, d, cs);
	if (r != RN_OK)
		return r;
	RNB_CUDA(cudaMemcpyAsync(accum, d, bytes, cudaMemcpyDeviceToHost, cs));
	return finish_sync(scene, cs, "rn_pt_render_accumulate");
}

rn_status rn_pt_autotune(rn_scene *scene, const rn_pt_camera *camera, const rn_pt_settings *settings, unsigned flags,
                         rn_pt_tuning *out) {
	TraceRange trace_range("rn_pt_autotune");
	PhysScene ps;
	PhysCamera pc;
	PhysSettings pst;
	rn_status r = make_phys_inputs(scene, camera, settings, flags, ps, pc, pst);
	if (r != RN_OK)
		return r;
	rn_pt_tuning t{};
	r = autotune_scene(scene, ps, pc, pst, t);
	if (r != RN_OK)
		return r;
	if (out)
		*out = t;
	return RN_OK;
}

rn_status rn_pt_count_traversal(rn_scene *scene, const rn_pt_camera *camera, const rn_pt_settings *settings,
                                long long *counters) {
	PhysScene ps;
	PhysCamera pc;
	PhysSettings pst;
	rn_status r = make_phys_inputs(scene, camera, settings, 0, ps, pc, pst);
	if (r != RN_OK)
		return r;
	if (!counters) {
		set_last_error("rn_pt_count_traversal: NULL counters");
		return RN_ERR_INVALID_ARGUMENT;
	}
	cudaStream_t cs = scene->stream;
	std::lock_guard<std::mutex> lock(scene->scratch_mu);
	RNB_CUDA(scene->scratch.ensure(256));
	unsigned long long *d = scene->scratch.as<unsigned long long>();
	RNB_CUDA(launch_count(ps, pc, pst, d, scene->d_status.as<int>(), cs));
	RNB_CUDA(cudaMemcpyAsync(counters, d, 7 * sizeof(long long), cudaMemcpyDeviceToHost, cs));
	return finish_sync(scene, cs, "rn_pt_count_traversal");
}

rn_status rn_pt_render(rn_scene *scene, const rn_pt_camera *camera, const rn_pt_settings *settings, unsigned flags,
                       void *stream, float *rgb) {
	TraceRange trace_range("rn_pt_render");
	PhysScene ps;
	PhysCamera pc;
	PhysSettings pst;
	rn_status r = make_phys_inputs(scene, camera, settings, flags, ps, pc, pst);
	if (r != RN_OK)
		return r;
	if (!rgb) {
		set_last_error("rn_pt_render: NULL rgb");
		return RN_ERR_INVALID_ARGUMENT;
	}
	cudaStream_t cs = pick_stream(scene, stream);
	const long nf = static_cast<long>(camera->width) * camera->height * 3;
	const size_t bytes = static_cast<size_t>(nf) * sizeof(float);
	const float inv = settings->spp > 0 ? 1.0f / static_cast<float>(settings->spp) : 0.0f;
	const bool dev = (flags & RN_PT_DEVICE_POINTERS) != 0;
	std::unique_lock<std::mutex> lock(scene->scratch_mu, std::defer_lock);
	float *acc;
	if (dev) {
		RNB_CUDA(scene->accum.ensure(bytes));
		acc = scene->accum.as<float>();
	} else {
		lock.lock();
		RNB_CUDA(scene->scratch.ensure(2 * bytes + 256));
		acc = scene->scratch.as<float>();
	}
	RNB_CUDA(cudaMemsetAsync(acc, 0, bytes, cs));
	r = run_integrator(scene, settings, flags, ps, pc, pst, acc, cs);
	if (r != RN_OK)
		return r;
	if (dev) {
		RNB_CUDA(launch_resolve(acc, rgb, nf, inv, cs));
		return RN_OK;
	}
	float *mean = acc + nf + 64;
	RNB_CUDA(launch_resolve(acc, mean, nf, inv, cs));
	RNB_CUDA(cudaMemcpyAsync(rgb, mean, bytes, cudaMemcpyDeviceToHost, cs));
	return finish_sync(scene, cs, "rn_pt_render");
}

} // extern "C"
