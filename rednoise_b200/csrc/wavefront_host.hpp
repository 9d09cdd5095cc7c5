// Host side of the wavefront integrator: pools, job tables, wave schedule and
// the CUDA graph that replays a whole frame.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"
#include "wavefront.cuh"

namespace rnb {

void wf_grid_sizes(int &grid_ext, int &grid_shade, int &grid_sh, int &grid_dyn, int &grid_bin);

// Samples per wave that keep about 2^20 paths in flight (at least 1, at most spp).
inline int default_samples_per_wave(long n_pix, int spp) {
	long k = n_pix > 0 ? (1L << 20) / n_pix : 1;
	if (k < 1)
		k = 1;
	if (k > spp)
		k = spp;
	return static_cast<int>(k < 1 ? 1 : k);
}

// Device bytes per wavefront path slot: origin, direction, throughput, radiance,
// pixel, sample, hit record, two queues and the sorted queue, the two parts of the bin
// key, the first-level sorted queue with its fine keys, shadow record with the two
// parts of its key and its sorted position.
constexpr size_t kWfBytesPerPath = 4 * 16 + 4 * 4 + 3 * 4 + 2 + 1 + 4 + 1 + 3 * 16 + 2 + 1 + 4;
// Adjoint waves add per slot: the list (32 B per entry), its length and the shadow
// record's two gradient float4s.
inline size_t wf_adjoint_bytes_per_path(int list_entries) {
	return kWfBytesPerPath + 32 * static_cast<size_t>(list_entries) + 4 + 32;
}

// Memory the autotuners let a path pool take: half the free device memory, at most 32 GiB.
inline cudaError_t wf_pool_budget(size_t &budget) {
	size_t free_b = 0, total_b = 0;
	const cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
	budget = free_b / 2 < (static_cast<size_t>(32) << 30) ? free_b / 2 : (static_cast<size_t>(32) << 30);
	return e;
}

class WfContext {
public:
	~WfContext();
	// Set up pools, job table and the wave schedule for these jobs (host copies
	// of the job descriptors; their accum pointers are device pointers). Each wave
	// holds `spw` samples of every pixel of every active job.
	rn_status configure(const std::vector<WfJob> &jobs, int max_depth, int order, int spw, cudaStream_t st);
	// Optional frame prologue / epilogue captured with the waves: zero the
	// accumulators first, then write means = sums * inv_spp per segment.
	struct Resolve {
		const float *accum;
		float *mean;
		long n_floats;
		float inv_spp;
	};
	void set_frame_io(float *zero_ptr, size_t zero_bytes, const std::vector<Resolve> &resolves);
	// Enqueue every wave of the frame on st (direct launches); with a clock, an event
	// is recorded before the frame and after every stage.
	rn_status enqueue(int *status, cudaStream_t st, WfStageClock *clock = nullptr);
	// Capture the frame into a CUDA graph on first use, then launch it.
	rn_status launch_graph(int *status, cudaStream_t st);
	int capacity() const { return capacity_; }
	// Traversal stages with per-lane ray replacement (1, default) or one ray per lane (0).
	void set_dynamic(int dyn) {
		if (dyn != dyn_)
			release_graph();
		dyn_ = dyn;
	}
	int dynamic() const { return dyn_; }
	// Binning sort of the closest-hit queues after the first bounce (1) or none (0, default).
	void set_sort(int sort) {
		if (sort != sort_)
			release_graph();
		sort_ = sort;
	}
	int sort() const { return sort_; }
	// Adjoint waves (path replay backpropagation): list_entries continuation vertices
	// per path (max_depth - 1 suffice), gradients added to d_alb / d_em (device, 3 floats
	// per triangle). Takes effect at the next configure; run them with enqueue.
	void set_adjoint(int list_entries, float *d_alb, float *d_em) {
		release_graph();
		adj_entries_ = list_entries;
		d_alb_ = d_alb;
		d_em_ = d_em;
	}

private:
	rn_status ensure_pool(int capacity);
	rn_status ensure_adjoint();
	void release_graph();

	DevBuf o_, d_, beta_, L_, pixel_, sample_, hit_idx_, hit_t_, q0_, q1_, sh_o_, sh_d_, sh_c_, counters_;
	DevBuf keys_, fine_, sorted_coarse_, sorted_fine_, sorted_, bins_, bin_hist_, sh_keys_, sh_fine_, sh_sorted_;
	DevBuf adj_pt_, adj_dlog_, adj_n_, sh_gdlog_, sh_gle_;
	DevBuf d_jobs_, d_wave_tab_;
	WfPool pool_{};
	int adj_entries_ = 0;
	float *d_alb_ = nullptr, *d_em_ = nullptr;
	int capacity_ = 0;
	int max_depth_ = 0;
	int order_ = 0;
	int grid_ext_ = 0, grid_shade_ = 0, grid_sh_ = 0, grid_dyn_ = 0, grid_bin_ = 0;
	int dyn_ = 1;
	int sort_ = 0;
	std::vector<WfWave> waves_;
	std::vector<WfJob> host_jobs_; // staging copies kept alive for the asynchronous uploads
	std::vector<int> host_tab_;
	std::vector<long> key_;
	float *zero_ptr_ = nullptr;
	size_t zero_bytes_ = 0;
	std::vector<Resolve> resolves_;
	cudaGraph_t graph_ = nullptr;
	cudaGraphExec_t exec_ = nullptr;
	int *graph_status_ = nullptr;
};

} // namespace rnb
