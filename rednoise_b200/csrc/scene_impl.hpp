// The opaque rn_scene behind both C ABIs.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "host_scene.hpp"
#include "traverse.cuh"
#include "wavefront_host.hpp"

// Per-triangle shading records, indexed by original triangle index.
//  ref:  (normal.xyz, reference Material as int bits), (r, g, b in 0..255, roughness)
//  phys: (albedo.rgb, physical material as int bits), (Le.rgb, GGX alpha or IOR)
struct rn_scene {
	rnb::TriangleSet tris;
	std::mutex mu;
	bool host_built = false;
	bool prepared = false;
	rnb::Bvh2 bvh;
	int internal_nodes = 0;
	double build_ms = 0.0;

	int device = -1;
	cudaStream_t stream = nullptr;
	rnb::DevBuf d_nodes, d_nodes4, d_tris, d_ref_shade, d_phys_shade, d_emitters;
	rnb::DevBuf d_ref_geom; // ray-traced renderer: vertices and vertex normals, uploaded on first use
	// GPU-built linear BVH (rn_pt_scene_build_lbvh), selected by RN_PT_LBVH
	rnb::DevBuf d_lbvh_nodes, d_lbvh_tris;
	rnb::SceneView lbvh_view{};
	bool lbvh_ready = false;
	int lbvh_depth = 0;
	bool ref_geom_ready = false;
	rnb::DevBuf d_status; // error word for asynchronous (device-pointer) calls
	rnb::SceneView view{};
	int n_emitters = 0;
	float emit_area_total = 0.0f;

	// Scratch for host-pointer calls (rays in, results out).
	std::mutex scratch_mu;
	rnb::DevBuf scratch;
	// Work counter of the persistent kernels and the accumulator of
	// device-pointer renders (calls on one scene are serialised on its stream).
	rnb::DevBuf d_counter;
	rnb::DevBuf accum;
	rnb::DevBuf adj; // view table and gradient buffers of device-pointer adjoint calls
	rnb::DevBuf d_adj_counter; // work counter of the adjoint kernel
	// Wavefront pools and the captured frame graph of single-scene renders.
	std::unique_ptr<rnb::WfContext> wf;
	std::unique_ptr<rnb::WfContext> wf_adj; // the wavefront adjoint's pools and schedule
	// Autotuner choices per (width, height, max_depth, order):
	// (integrator, samples per wave, per-lane ray replacement).
	std::map<std::tuple<int, int, int, int>, std::tuple<int, int, int, int>> tuned;
	rnb::DevBuf tune_accum;

	~rn_scene();
};

namespace rnb {

// Host BVH build only (caller holds s->mu).
rn_status build_host(rn_scene *s);
// Build the BVH and upload everything (idempotent, thread safe).
rn_status prepare_scene(rn_scene *s);

// Resolve the stream for a call: the caller's or the scene's own.
inline cudaStream_t pick_stream(rn_scene *s, void *stream) {
	return stream ? static_cast<cudaStream_t>(stream) : s->stream;
}

// Kernel launchers (trace_kernels.cu).
cudaError_t launch_trace_closest(const SceneView &v, int n, const float *o, const float *d, const int *ignore,
                                 int order, int *tri, float *t, float *u, float *vv, int *err, cudaStream_t st);
cudaError_t launch_trace_any(const SceneView &v, int n, const float *o, const float *d, const float *tmax,
                             const int *ignore, int *occ, int *err, cudaStream_t st);

} // namespace rnb
