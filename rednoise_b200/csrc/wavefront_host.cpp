#include "wavefront_host.hpp"

#include <algorithm>

#include "pt_kernels.hpp"

namespace rnb {

WfContext::~WfContext() { release_graph(); }

void WfContext::release_graph() {
	if (exec_)
		cudaGraphExecDestroy(exec_);
	if (graph_)
		cudaGraphDestroy(graph_);
	exec_ = nullptr;
	graph_ = nullptr;
	graph_status_ = nullptr;
}

rn_status WfContext::ensure_pool(int capacity) {
	if (capacity <= capacity_)
		return RN_OK;
	release_graph();
	// The buffers grow one by one and a grown buffer frees its old memory: until
	// all of them have grown, the pool describes no usable capacity.
	capacity_ = 0;
	const size_t n = static_cast<size_t>(capacity);
	RNB_CUDA(o_.ensure(n * 16));
	RNB_CUDA(d_.ensure(n * 16));
	RNB_CUDA(beta_.ensure(n * 16));
	RNB_CUDA(L_.ensure(n * 16));
	RNB_CUDA(pixel_.ensure(n * 4));
	RNB_CUDA(sample_.ensure(n * 4));
	RNB_CUDA(hit_idx_.ensure(n * 4));
	RNB_CUDA(hit_t_.ensure(n * 4));
	RNB_CUDA(q0_.ensure(n * 4));
	RNB_CUDA(q1_.ensure(n * 4));
	RNB_CUDA(sh_o_.ensure(n * 16));
	RNB_CUDA(sh_d_.ensure(n * 16));
	RNB_CUDA(sh_c_.ensure(n * 16));
	RNB_CUDA(counters_.ensure(kCntTotal * sizeof(unsigned)));
	RNB_CUDA(keys_.ensure(n * sizeof(uint16_t)));
	RNB_CUDA(fine_.ensure(n));
	RNB_CUDA(sorted_coarse_.ensure(n * 4));
	RNB_CUDA(sorted_fine_.ensure(n));
	RNB_CUDA(sorted_.ensure(n * 4));
	RNB_CUDA(bins_.ensure(2 * kBins * sizeof(unsigned)));
	RNB_CUDA(bin_hist_.ensure(static_cast<size_t>(kBinBlocksMax) * kBins * sizeof(unsigned)));
	RNB_CUDA(sh_keys_.ensure(n * sizeof(uint16_t)));
	RNB_CUDA(sh_fine_.ensure(n));
	RNB_CUDA(sh_sorted_.ensure(n * 4));
	pool_.o = o_.as<float4>();
	pool_.d = d_.as<float4>();
	pool_.beta = beta_.as<float4>();
	pool_.L = L_.as<float4>();
	pool_.pixel = pixel_.as<uint32_t>();
	pool_.sample = sample_.as<uint32_t>();
	pool_.hit_idx = hit_idx_.as<int>();
	pool_.hit_t = hit_t_.as<float>();
	pool_.rank = nullptr;
	pool_.queue[0] = q0_.as<int>();
	pool_.queue[1] = q1_.as<int>();
	pool_.sh_o = sh_o_.as<float4>();
	pool_.sh_d = sh_d_.as<float4>();
	pool_.sh_c = sh_c_.as<float4>();
	pool_.counters = counters_.as<unsigned>();
	pool_.keys = keys_.as<uint16_t>();
	pool_.fine = fine_.as<uint8_t>();
	pool_.sorted_coarse = sorted_coarse_.as<int>();
	pool_.sorted_fine = sorted_fine_.as<uint8_t>();
	pool_.sorted = sorted_.as<int>();
	pool_.bins = bins_.as<unsigned>();
	pool_.bin_hist = bin_hist_.as<unsigned>();
	pool_.sh_keys = sh_keys_.as<uint16_t>();
	pool_.sh_fine = sh_fine_.as<uint8_t>();
	pool_.sh_sorted = sh_sorted_.as<int>();
	pool_.capacity = capacity;
	capacity_ = capacity;
	return RN_OK;
}

rn_status WfContext::ensure_adjoint() {
	pool_.adj_pt = pool_.adj_dlog = pool_.sh_gdlog = pool_.sh_gle = nullptr;
	pool_.adj_n = nullptr;
	pool_.adj_entries = 0;
	pool_.d_alb = pool_.d_em = nullptr;
	if (adj_entries_ <= 0)
		return RN_OK;
	const size_t n = static_cast<size_t>(capacity_);
	const size_t m = n * static_cast<size_t>(adj_entries_);
	RNB_CUDA(adj_pt_.ensure(m * 16));
	RNB_CUDA(adj_dlog_.ensure(m * 16));
	RNB_CUDA(adj_n_.ensure(n * 4));
	RNB_CUDA(sh_gdlog_.ensure(n * 16));
	RNB_CUDA(sh_gle_.ensure(n * 16));
	pool_.adj_pt = adj_pt_.as<float4>();
	pool_.adj_dlog = adj_dlog_.as<float4>();
	pool_.adj_n = adj_n_.as<int>();
	pool_.sh_gdlog = sh_gdlog_.as<float4>();
	pool_.sh_gle = sh_gle_.as<float4>();
	pool_.adj_entries = adj_entries_;
	pool_.d_alb = d_alb_;
	pool_.d_em = d_em_;
	return RN_OK;
}

rn_status WfContext::configure(const std::vector<WfJob> &jobs, int max_depth, int order, int spw,
                               cudaStream_t st) {
	if (jobs.empty() || max_depth < 1 || max_depth > kWfMaxDepth || spw < 1) {
		set_last_error("wavefront: need at least one job, 1 <= max_depth <= 64 and samples per wave >= 1");
		return RN_ERR_INVALID_ARGUMENT;
	}
	// Same frame structure as the captured graph: only the job table changes
	// (sample offsets, seeds, accumulators), which the kernels read from memory.
	std::vector<long> key = {static_cast<long>(jobs.size()), max_depth, order, spw};
	for (const WfJob &j : jobs) {
		key.push_back(j.n_pix);
		key.push_back(j.spp);
	}
	if (exec_ && key == key_) {
		host_jobs_ = jobs;
		RNB_CUDA(cudaMemcpyAsync(d_jobs_.p, host_jobs_.data(), jobs.size() * sizeof(WfJob), cudaMemcpyHostToDevice,
		                         st));
		return RN_OK;
	}
	release_graph();
	key_ = key;
	int max_spp = 0;
	for (const WfJob &j : jobs)
		max_spp = std::max(max_spp, j.spp);
	const int n_waves = (max_spp + spw - 1) / spw;
	// Wave schedule: wave w holds samples [w*spw, (w+1)*spw) of every job that has them.
	std::vector<int> tab;
	struct Span {
		size_t off;
		int n_jobs;
		long n_slots, n_pix;
		int only_job;
	};
	std::vector<Span> spans;
	long capacity = 1;
	for (int w = 0; w < n_waves; w++) {
		std::vector<int> ids, bases, pbases, nsamp;
		long base = 0, pbase = 0;
		for (size_t j = 0; j < jobs.size(); j++) {
			const int k = std::min(spw, jobs[j].spp - w * spw);
			if (k <= 0 || jobs[j].n_pix <= 0)
				continue;
			ids.push_back(static_cast<int>(j));
			bases.push_back(static_cast<int>(base));
			pbases.push_back(static_cast<int>(pbase));
			nsamp.push_back(k);
			base += static_cast<long>(k) * jobs[j].n_pix;
			pbase += jobs[j].n_pix;
			if (base > (1L << 30)) {
				set_last_error("wavefront: more than 2^30 paths in one wave");
				return RN_ERR_CAPACITY;
			}
		}
		spans.push_back({tab.size(), static_cast<int>(ids.size()), base, pbase, ids.size() == 1 ? ids[0] : -1});
		for (const auto *v : {&ids, &bases, &pbases, &nsamp})
			tab.insert(tab.end(), v->begin(), v->end());
		capacity = std::max(capacity, base);
	}
	rn_status r = ensure_pool(static_cast<int>(capacity));
	if (r != RN_OK)
		return r;
	r = ensure_adjoint();
	if (r != RN_OK)
		return r;
	if (grid_ext_ == 0)
		wf_grid_sizes(grid_ext_, grid_shade_, grid_sh_, grid_dyn_, grid_bin_);
	host_jobs_ = jobs;
	host_tab_ = tab;
	RNB_CUDA(d_jobs_.ensure(jobs.size() * sizeof(WfJob)));
	RNB_CUDA(d_wave_tab_.ensure(std::max<size_t>(tab.size(), 1) * sizeof(int)));
	RNB_CUDA(cudaMemcpyAsync(d_jobs_.p, host_jobs_.data(), jobs.size() * sizeof(WfJob), cudaMemcpyHostToDevice, st));
	if (!tab.empty())
		RNB_CUDA(cudaMemcpyAsync(d_wave_tab_.p, host_tab_.data(), tab.size() * sizeof(int), cudaMemcpyHostToDevice,
		                         st));
	waves_.clear();
	const int *t = d_wave_tab_.as<int>();
	for (int w = 0; w < n_waves; w++) {
		const Span &sp = spans[static_cast<size_t>(w)];
		WfWave wv;
		wv.jobs = t + sp.off;
		wv.bases = wv.jobs + sp.n_jobs;
		wv.pbases = wv.bases + sp.n_jobs;
		wv.nsamp = wv.pbases + sp.n_jobs;
		wv.n_jobs = sp.n_jobs;
		wv.n_slots = static_cast<int>(sp.n_slots);
		wv.n_pix = static_cast<int>(sp.n_pix);
		wv.first_sample = w * spw;
		wv.only_job = sp.only_job;
		waves_.push_back(wv);
	}
	max_depth_ = max_depth;
	order_ = order;
	return RN_OK;
}

void WfContext::set_frame_io(float *zero_ptr, size_t zero_bytes, const std::vector<Resolve> &resolves) {
	bool same = zero_ptr == zero_ptr_ && zero_bytes == zero_bytes_ && resolves.size() == resolves_.size();
	for (size_t i = 0; same && i < resolves.size(); i++)
		same = resolves[i].accum == resolves_[i].accum && resolves[i].mean == resolves_[i].mean &&
		       resolves[i].n_floats == resolves_[i].n_floats && resolves[i].inv_spp == resolves_[i].inv_spp;
	if (!same)
		release_graph();
	zero_ptr_ = zero_ptr;
	zero_bytes_ = zero_bytes;
	resolves_ = resolves;
}

rn_status WfContext::enqueue(int *status, cudaStream_t st, WfStageClock *clock) {
	if (clock) {
		if (!clock->start)
			RNB_CUDA(cudaEventCreate(&clock->start));
		RNB_CUDA(cudaEventRecord(clock->start, st));
	}
	if (zero_ptr_ && zero_bytes_)
		RNB_CUDA(cudaMemsetAsync(zero_ptr_, 0, zero_bytes_, st));
	const WfLaunch lc{grid_ext_, grid_shade_, grid_sh_, grid_dyn_, grid_bin_, dyn_, sort_, clock};
	for (const WfWave &w : waves_)
		RNB_CUDA(wf_launch_wave(d_jobs_.as<WfJob>(), pool_, w, max_depth_, order_, lc, status, st));
	for (const Resolve &r : resolves_)
		RNB_CUDA(launch_resolve(r.accum, r.mean, r.n_floats, r.inv_spp, st));
	if (clock && !resolves_.empty())
		RNB_CUDA(clock->mark(kStAccumulate, static_cast<int>(resolves_.size()), st));
	return RN_OK;
}

rn_status WfContext::launch_graph(int *status, cudaStream_t st) {
	if (exec_ && graph_status_ != status)
		release_graph();
	if (!exec_) {
		RNB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
		rn_status r = enqueue(status, st);
		cudaGraph_t g = nullptr;
		cudaError_t e = cudaStreamEndCapture(st, &g);
		if (r != RN_OK) {
			if (g)
				cudaGraphDestroy(g);
			return r;
		}
		RNB_CUDA(e);
		graph_ = g;
		RNB_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
		graph_status_ = status;
	}
	RNB_CUDA(cudaGraphLaunch(exec_, st));
	return RN_OK;
}

} // namespace rnb
