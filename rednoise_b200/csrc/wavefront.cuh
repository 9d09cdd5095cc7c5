// Wavefront integrator: path state in structure-of-arrays pools, one kernel
// per stage, device-side queues with warp-aggregated appends.
//
// A "wave" holds one sample of every pixel of every active job (a job is one
// scene + camera + settings; a single render is a batch of one job). Stages per
// bounce k (k = 0 .. max_depth-1), all launched with a fixed persistent grid
// that reads its queue length from device memory, so the whole per-frame
// sequence can be captured once as a CUDA graph:
//   extend  : closest hit for every queued ray        (traversal only, few registers)
//   shade   : vertex shading, NEE shadow-ray append, continuation append
//   shadow  : any-hit for every shadow record, radiance added to the path
// then `accumulate` adds each path's radiance to its pixel sum. Samples are
// added in sample order per pixel, so results equal the megakernel's.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "physical.cuh"

namespace rnb {

constexpr int kWfMaxDepth = 64;

struct WfJob {
	PhysScene sc;
	PhysCamera cam;
	PhysSettings st;
	float *accum; // 3 floats per pixel (sums); unused by adjoint waves
	int n_pix;
	int spp;
	const float *dimg = nullptr; // adjoint waves: dL/d(mean image), 3 floats per pixel
};

// Pools of `capacity` path slots.
struct WfPool {
	float4 *o;    // origin.xyz, ignore (int bits)
	float4 *d;    // direction.xyz, prev_pdf
	float4 *beta; // throughput.xyz, bounce (int bits)
	float4 *L;    // radiance.xyz, job (int bits)
	uint32_t *pixel;
	uint32_t *sample;
	int *hit_idx;
	float *hit_t;
	int *rank;     // hit rank (unused by shading; kept for the closest-hit record)
	int *queue[2]; // ray queues, alternating by bounce parity
	float4 *sh_o;  // shadow origin.xyz, tmax
	float4 *sh_d;  // shadow direction.xyz, ignore (int bits)
	float4 *sh_c;  // contribution.xyz, slot (int bits)
	// counters: [0, kWfMaxDepth] ray-queue lengths per bounce, [kWfMaxDepth+1 ...] shadow
	// lengths per bounce, then per-bounce fetch counters of extend and shadow.
	unsigned *counters;
	// Ray binning (optional): the shade stage writes each continuation ray's bin in
	// two parts, keys (the 15-bit Morton cell of its origin, 5 bits per axis over the
	// scene's box) and fine (a 16 x 16 octahedral cell of its direction). Before the
	// next closest-hit stage a counting sort by origin cell writes the queue to
	// sorted_coarse (carrying each entry's direction cell to sorted_fine), and a
	// counting sort of every origin cell's entries by direction cell writes it to
	// sorted: the lanes of a warp then trace rays that start close together in
	// similar directions and visit the same nodes.
	uint16_t *keys;
	uint8_t *fine;
	int *sorted_coarse;
	uint8_t *sorted_fine;
	int *sorted;
	unsigned *bins;     // kBins bin totals, then kBins exclusive bin starts
	unsigned *bin_hist; // kBinBlocksMax rows of kBins: per-block counts, then per-block offsets
	// With binning on, each shadow record's key in two parts (the 15-bit Morton cell
	// of its origin, the shading point, and the 6-bit Morton sub-cell of the origin
	// inside it) and the shadow stage's order sorted by them (the same two counting
	// sorts, with sorted_coarse and sorted_fine as scratch).
	uint16_t *sh_keys;
	uint8_t *sh_fine;
	int *sh_sorted;
	// Adjoint waves only (null otherwise; path replay backpropagation). Per slot, the
	// list of its continuation vertices, entry e of slot s at e * capacity + s:
	// adj_pt = radiance gathered up to and including the vertex (written by the
	// next shade stage, when the vertex's next-event term is in), adj_dlog = d log
	// (continuation weight) / d albedo .xyz and the vertex's triangle (int bits);
	// adj_n = entries per slot. Per shadow record, sh_gdlog = d log f(light) / d albedo
	// .xyz and the scattering triangle, sh_gle = the sampled emitter's radiance .xyz
	// and the emitter triangle. d_alb / d_em: the gradients (3 floats per triangle).
	float4 *adj_pt;
	float4 *adj_dlog;
	int *adj_n;
	float4 *sh_gdlog;
	float4 *sh_gle;
	float *d_alb;
	float *d_em;
	int adj_entries; // list entries per slot (>= max_depth - 1)
	int capacity;
};

constexpr int kBinBits = 15;
constexpr int kBins = 1 << kBinBits;
constexpr int kBinBlocksMax = 256; // blocks of the counting sorts

constexpr int kCntRays = 0;
constexpr int kCntShadow = kWfMaxDepth + 1;
constexpr int kCntFetchExt = 2 * (kWfMaxDepth + 1);
constexpr int kCntFetchSh = 3 * (kWfMaxDepth + 1);
constexpr int kCntTotal = 4 * (kWfMaxDepth + 1);

// One wave's generation table. A wave holds `spw` consecutive samples of every
// pixel of each active job, laid out sample-major per job:
//   slot = bases[a] + k * n_pix + pixel,  k < nsamp[a]
// and is accumulated per pixel over k in sample order.
struct WfWave {
	const int *jobs;    // active job ids
	const int *bases;   // first slot of each active job
	const int *pbases;  // first accumulate index of each active job
	const int *nsamp;   // samples of each active job in this wave
	int n_jobs;
	int n_slots;        // paths in the wave
	int n_pix;          // pixels in the wave (sum of active jobs' pixels)
	int first_sample;   // sample index of k = 0, relative to each job's sample_offset
	int only_job;       // the job id when the wave holds one job, else -1
};

// Launch shapes and stage options of a wave.
// Stage kinds of a frame, for per-stage timing.
enum WfStage : int {
	kStCamera = 0,
	kStRaySort,    // two-level counting sort of a bounce's closest-hit queue
	kStExtend,     // closest hits
	kStShade,      // shading, next-event records, continuation
	kStShadowSort, // counting sort of a bounce's shadow records
	kStShadow,     // any hits of the shadow records
	kStAccumulate, // per-pixel sums and the frame's resolve
	kStCount
};

// CUDA events recorded after every stage of a frame launched directly (not from
// the captured graph): consecutive events bracket one stage each. Host-side; the
// events are created on first use and destroyed with the clock.
struct WfStageClock {
	static constexpr int kMax = 4096;
	cudaEvent_t start = nullptr;
	cudaEvent_t ev[kMax] = {};
	int kind[kMax] = {};
	int n = 0;
	int launches = 0; // kernels launched in the frame
	bool overflow = false;
	cudaError_t mark(int stage, int kernels, cudaStream_t st) {
		launches += kernels;
		if (n >= kMax) {
			overflow = true;
			return cudaSuccess;
		}
		if (!ev[n]) {
			const cudaError_t e = cudaEventCreate(&ev[n]);
			if (e != cudaSuccess)
				return e;
		}
		kind[n] = stage;
		return cudaEventRecord(ev[n++], st);
	}
	~WfStageClock() {
		if (start)
			cudaEventDestroy(start);
		for (int i = 0; i < kMax; i++)
			if (ev[i])
				cudaEventDestroy(ev[i]);
	}
};

struct WfLaunch {
	int grid_ext, grid_shade, grid_sh, grid_dyn, grid_bin;
	int dyn;  // traversal stages use persistent warps that replace finished rays per lane
	int sort; // closest-hit queues after the first bounce are binned by origin and direction
	WfStageClock *clock = nullptr; // per-stage events (profiled frames only)
};

cudaError_t wf_launch_wave(const WfJob *d_jobs, const WfPool &pool, const WfWave &wave, int max_depth, int order,
                           const WfLaunch &lc, int *status, cudaStream_t st);

} // namespace rnb
