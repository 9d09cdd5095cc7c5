// Batched rendering of many jobs (scene + camera + settings) per launch.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "pt_kernels.hpp"
#include "render_impl.hpp"
#include "scene_impl.hpp"
#include "trace_range.hpp"

struct rn_pt_batch {
	std::vector<rn_pt_job> jobs;
	std::vector<rnb::WfJob> wf_jobs; // kernel inputs, accum pointers into `accum`
	std::vector<long> offsets;       // float offset of each job's image in accum / mean
	rnb::DevBuf accum, mean, status;
	rnb::WfContext wf;
	cudaStream_t stream = nullptr;
	int integrator = RN_PT_WAVEFRONT;
	int order = 0;
	int max_depth = 1;
	int spw = 1;
	int forced_sort = -1; // RN_PT_RAY_SORT / RN_PT_NO_RAY_SORT at creation: 1 / 0; else tuned
	long total_floats = 0;
	~rn_pt_batch() {
		if (stream)
			cudaStreamDestroy(stream);
	}
};

using namespace rnb;

namespace {

// spp_div > 1 (autotuning probes only): every job renders ceil(spp / spp_div) samples.
rn_status batch_enqueue(rn_pt_batch *b, unsigned sample_offset, cudaStream_t cs, int spp_div = 1) {
	std::vector<WfJob> jobs = b->wf_jobs;
	for (size_t i = 0; i < jobs.size(); i++) {
		jobs[i].st.sample_offset = b->jobs[i].settings.sample_offset + sample_offset;
		if (spp_div > 1) {
			jobs[i].spp = (jobs[i].spp + spp_div - 1) / spp_div;
			jobs[i].st.spp = jobs[i].spp;
		}
	}
	int *status = b->status.as<int>();
	if (b->integrator == RN_PT_WAVEFRONT) {
		rn_status r = b->wf.configure(jobs, b->max_depth, b->order, b->spw, cs);
		if (r != RN_OK)
			return r;
		return b->wf.launch_graph(status, cs);
	}
	// Plain GPU baseline: one megakernel launch per job.
	RNB_CUDA(cudaMemsetAsync(b->accum.p, 0, static_cast<size_t>(b->total_floats) * sizeof(float), cs));
	for (size_t i = 0; i < jobs.size(); i++) {
		rn_scene *s = b->jobs[i].scene;
		RNB_CUDA(s->d_counter.ensure(256));
		RNB_CUDA(launch_megakernel(jobs[i].sc, jobs[i].cam, jobs[i].st, jobs[i].accum, s->d_counter.as<unsigned>(),
		                           status, cs));
		const long nf = static_cast<long>(jobs[i].n_pix) * 3;
		RNB_CUDA(launch_resolve(jobs[i].accum, b->mean.as<float>() + b->offsets[i], nf,
		                        jobs[i].spp > 0 ? 1.0f / static_cast<float>(jobs[i].spp) : 0.0f, cs));
	}
	return RN_OK;
}

// Time one frame of each candidate at the batch's own image sizes (with a quarter
// of every job's samples once the largest job has 16 or more) and keep the fastest:
// one megakernel per job; the wavefront without and with ray binning at the default
// queue capacity; then the better of those at 2x, 4x, ... the capacity while that
// keeps helping, up to the probe's largest spp, within a memory budget.
rn_status autotune_batch(rn_pt_batch *b, int max_spp, long total_pix) {
	const int div = max_spp >= 16 ? 4 : 1;
	const int probe_spp = (max_spp + div - 1) / div;
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
	auto time_one = [&](int integ, int sort, int spw, float &ms) -> rn_status {
		b->integrator = integ;
		b->wf.set_sort(sort);
		b->spw = spw;
		rn_status r = batch_enqueue(b, 0x40000000u, b->stream, div); // warm-up (and graph capture)
		if (r != RN_OK)
			return r;
		RNB_CUDA(cudaEventRecord(ev.a, b->stream));
		r = batch_enqueue(b, 0x40000000u, b->stream, div);
		if (r != RN_OK)
			return r;
		RNB_CUDA(cudaEventRecord(ev.b, b->stream));
		RNB_CUDA(cudaEventSynchronize(ev.b));
		RNB_CUDA(cudaEventElapsedTime(&ms, ev.a, ev.b));
		return RN_OK;
	};
	const int spw0 = b->spw;
	float best = 0.0f;
	int pick = RN_PT_MEGAKERNEL, pick_sort = 0, pick_spw = spw0;
	rn_status r = time_one(RN_PT_MEGAKERNEL, 0, spw0, best);
	if (r != RN_OK)
		return r;
	float best_wf = 0.0f;
	int wf_sort = 0;
	for (int sort : {0, 1}) {
		if (b->forced_sort >= 0 && sort != b->forced_sort)
			continue;
		float ms = 0.0f;
		r = time_one(RN_PT_WAVEFRONT, sort, spw0, ms);
		if (r != RN_OK)
			return r;
		if (best_wf == 0.0f || ms < best_wf) {
			best_wf = ms;
			wf_sort = sort;
		}
	}
	int wf_spw = spw0;
	size_t budget = 0;
	RNB_CUDA(wf_pool_budget(budget));
	for (int spw = 2 * spw0; spw <= probe_spp; spw *= 2) {
		if (static_cast<size_t>(total_pix) * spw * kWfBytesPerPath > budget)
			break;
		float ms = 0.0f;
		r = time_one(RN_PT_WAVEFRONT, wf_sort, spw, ms);
		if (r != RN_OK)
			return r;
		if (ms >= best_wf)
			break;
		best_wf = ms;
		wf_spw = spw;
	}
	if (best_wf < best) {
		pick = RN_PT_WAVEFRONT;
		pick_sort = wf_sort;
		pick_spw = wf_spw;
	}
	b->integrator = pick;
	b->wf.set_sort(pick_sort);
	b->spw = pick_spw;
	return RN_OK;
}

} // namespace

extern "C" {

rn_status rn_pt_batch_create(const rn_pt_job *jobs, int n, int integrator, unsigned flags, rn_pt_batch **out) {
	TraceRange trace_range("rn_pt_batch_create");
	if (!jobs || n <= 0 || !out) {
		set_last_error("rn_pt_batch_create: need n > 0 jobs and an output pointer");
		return RN_ERR_INVALID_ARGUMENT;
	}
	if (integrator != RN_PT_AUTO && integrator != RN_PT_MEGAKERNEL && integrator != RN_PT_WAVEFRONT) {
		set_last_error("rn_pt_batch_create: unknown integrator");
		return RN_ERR_INVALID_ARGUMENT;
	}
	*out = nullptr;
	std::unique_ptr<rn_pt_batch> b(new (std::nothrow) rn_pt_batch());
	if (!b)
		return RN_ERR_OUT_OF_MEMORY;
	b->jobs.assign(jobs, jobs + n);
	b->order = (flags & RN_PT_ORDER_NEAREST) ? kOrderNearest : kOrderReference;
	b->forced_sort = (flags & RN_PT_RAY_SORT) ? 1 : ((flags & RN_PT_NO_RAY_SORT) ? 0 : -1);
	if (b->forced_sort >= 0)
		b->wf.set_sort(b->forced_sort);
	long total = 0;
	int max_spp = 1;
	long max_pix = 1;
	for (int i = 0; i < n; i++) {
		PhysScene ps;
		PhysCamera pc;
		PhysSettings pst;
		rn_status r = make_phys_inputs(jobs[i].scene, &jobs[i].camera, &jobs[i].settings, flags, ps, pc, pst);
		if (r != RN_OK)
			return r;
		if (pst.max_depth > kWfMaxDepth) {
			set_last_error("rn_pt_batch_create: max_depth must be <= 64");
			return RN_ERR_INVALID_ARGUMENT;
		}
		WfJob j;
		j.sc = ps;
		j.cam = pc;
		j.st = pst;
		j.accum = nullptr;
		j.n_pix = pc.width * pc.height;
		j.spp = pst.spp;
		b->wf_jobs.push_back(j);
		b->offsets.push_back(total);
		total += static_cast<long>(j.n_pix) * 3;
		b->max_depth = std::max(b->max_depth, pst.max_depth);
		max_spp = std::max(max_spp, pst.spp);
		max_pix = std::max(max_pix, static_cast<long>(j.n_pix));
	}
	b->total_floats = total;
	RNB_CUDA(b->accum.ensure(static_cast<size_t>(total) * sizeof(float)));
	RNB_CUDA(b->mean.ensure(static_cast<size_t>(total) * sizeof(float)));
	RNB_CUDA(b->status.ensure(256));
	RNB_CUDA(cudaMemset(b->status.p, 0, 256));
	RNB_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
	for (int i = 0; i < n; i++)
		b->wf_jobs[i].accum = b->accum.as<float>() + b->offsets[i];
	// Paths per wave: about 2^20 in flight, counting every job's pixels.
	b->spw = default_samples_per_wave(total / 3, max_spp);
	std::vector<WfContext::Resolve> res;
	for (int i = 0; i < n; i++)
		res.push_back({b->wf_jobs[i].accum, b->mean.as<float>() + b->offsets[i],
		               static_cast<long>(b->wf_jobs[i].n_pix) * 3,
		               b->wf_jobs[i].spp > 0 ? 1.0f / static_cast<float>(b->wf_jobs[i].spp) : 0.0f});
	b->wf.set_frame_io(b->accum.as<float>(), static_cast<size_t>(total) * sizeof(float), res);
	if (integrator == RN_PT_AUTO) {
		rn_status r = autotune_batch(b.get(), max_spp, total / 3);
		if (r != RN_OK)
			return r;
	} else {
		b->integrator = integrator;
	}
	*out = b.release();
	return RN_OK;
}

rn_status rn_pt_batch_render(rn_pt_batch *b, unsigned sample_offset, unsigned flags, void *stream,
                             float *const *out) {
	TraceRange trace_range("rn_pt_batch_render");
	if (!b || !out) {
		set_last_error("rn_pt_batch_render: NULL argument");
		return RN_ERR_INVALID_ARGUMENT;
	}
	for (size_t i = 0; i < b->jobs.size(); i++)
		if (!out[i]) {
			set_last_error("rn_pt_batch_render: NULL output for a job");
			return RN_ERR_INVALID_ARGUMENT;
		}
	const bool dev = (flags & RN_PT_DEVICE_POINTERS) != 0;
	cudaStream_t cs = stream ? static_cast<cudaStream_t>(stream) : b->stream;
	rn_status r = batch_enqueue(b, sample_offset, cs);
	if (r != RN_OK)
		return r;
	for (size_t i = 0; i < b->jobs.size(); i++) {
		const size_t bytes = static_cast<size_t>(b->wf_jobs[i].n_pix) * 3 * sizeof(float);
		RNB_CUDA(cudaMemcpyAsync(out[i], b->mean.as<float>() + b->offsets[i], bytes,
		                         dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, cs));
	}
	if (dev)
		return RN_OK;
	int h = 0;
	RNB_CUDA(cudaMemcpyAsync(&h, b->status.p, sizeof(int), cudaMemcpyDeviceToHost, cs));
	RNB_CUDA(cudaStreamSynchronize(cs));
	if (h) {
		set_last_error("rn_pt_batch_render: device status word reports a traversal error");
		return RN_ERR_INTERNAL;
	}
	return RN_OK;
}

int rn_pt_batch_integrator(const rn_pt_batch *b) { return b ? b->integrator : -1; }

void rn_pt_batch_free(rn_pt_batch *b) { delete b; }

} // extern "C"
