// rn_scene lifetime, lazy device preparation and the ray-query entry points.
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "lbvh.hpp"
#include "scene_impl.hpp"
#include "trace_range.hpp"

namespace rnb {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string &msg) { g_last_error = msg; }
const char *get_last_error() { return g_last_error.c_str(); }

namespace {
std::atomic<long long> g_alloc_countdown{-1};
} // namespace

bool injected_allocation_failure() {
	long long v = g_alloc_countdown.load();
	while (v >= 0) {
		if (g_alloc_countdown.compare_exchange_weak(v, v - 1))
			return v == 0;
	}
	return false;
}

rn_status cuda_fail(cudaError_t e, const char *what) {
	set_last_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
	return e == cudaErrorMemoryAllocation ? RN_ERR_OUT_OF_MEMORY : RN_ERR_CUDA;
}

static float as_float(int i) {
	float f;
	std::memcpy(&f, &i, 4);
	return f;
}

rn_status build_host(rn_scene *s) {
	if (s->host_built)
		return RN_OK;
	const int n = static_cast<int>(s->tris.size());
	if (n <= 0) {
		set_last_error("scene has no triangles");
		return RN_ERR_INVALID_ARGUMENT;
	}
	if (n >= (1 << 28)) {
		set_last_error("scene has more than 2^28 triangles");
		return RN_ERR_CAPACITY;
	}
	auto t0 = std::chrono::steady_clock::now();
	build_reference_bvh(s->tris.v.data(), n, s->bvh);
	s->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
	s->host_built = true;
	return RN_OK;
}

rn_status prepare_scene(rn_scene *s) {
	TraceRange trace_range("scene prepare: BVH build and upload");
	std::lock_guard<std::mutex> lock(s->mu);
	if (s->prepared)
		return RN_OK;
	rn_status hs = build_host(s);
	if (hs != RN_OK)
		return hs;
	const int n = static_cast<int>(s->tris.size());
	int dev = 0;
	RNB_CUDA(cudaGetDevice(&dev));
	s->device = dev;
	auto t0 = std::chrono::steady_clock::now();
	DeviceLayout lay;
	flatten_bvh(s->tris, s->bvh, lay);
	s->build_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
	// Depth-first traversal with both children pushed needs at most depth + 1 slots.
	if (lay.depth + 1 > kStack) {
		set_last_error("BVH deeper than the traversal stack bound");
		return RN_ERR_CAPACITY;
	}
	s->internal_nodes = lay.internal_count;

	// Shading records indexed by original triangle.
	std::vector<F4> ref(static_cast<size_t>(n) * 2), phys(static_cast<size_t>(n) * 3);
	const TriangleSet &ts = s->tris;
	for (int i = 0; i < n; i++) {
		const size_t k = static_cast<size_t>(i);
		ref[2 * k] = {ts.normal[3 * k], ts.normal[3 * k + 1], ts.normal[3 * k + 2], as_float(ts.ref_material[k])};
		ref[2 * k + 1] = {static_cast<float>(ts.rgb[3 * k]), static_cast<float>(ts.rgb[3 * k + 1]),
		                  static_cast<float>(ts.rgb[3 * k + 2]), ts.roughness[k]};
		Vec3 ng = geometric_normal(&ts.v[9 * k]);
		phys[3 * k] = {ts.albedo[3 * k], ts.albedo[3 * k + 1], ts.albedo[3 * k + 2], as_float(ts.phys_material[k])};
		phys[3 * k + 1] = {ts.emission[3 * k], ts.emission[3 * k + 1], ts.emission[3 * k + 2], ts.phys_param[k]};
		phys[3 * k + 2] = {ng.x, ng.y, ng.z, 0.0f};
	}
	// The emitter flag marks the triangles that are in the light-sampling table.
	// Emitters (triangles with any Le > 0): (v0, tri), (e0, area), (e1, cumulative area).
	std::vector<F4> em;
	double acc = 0.0;
	for (int i = 0; i < n; i++) {
		const size_t k = static_cast<size_t>(i);
		if (ts.emission[3 * k] > 0.0f || ts.emission[3 * k + 1] > 0.0f || ts.emission[3 * k + 2] > 0.0f) {
			const float *t = &ts.v[9 * k];
			const double area = triangle_area(t);
			if (!(area > 0.0))
				continue; // a degenerate emitter can neither be hit nor sampled
			acc += area;
			phys[3 * k + 2].w = 1.0f;
			em.push_back({t[0], t[1], t[2], as_float(i)});
			em.push_back({t[3] - t[0], t[4] - t[1], t[5] - t[2], static_cast<float>(area)});
			em.push_back({t[6] - t[0], t[7] - t[1], t[8] - t[2], static_cast<float>(acc)});
		}
	}
	s->n_emitters = static_cast<int>(em.size() / 3);
	s->emit_area_total = static_cast<float>(acc);

	if (!s->stream)
		RNB_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
	auto up = [&](DevBuf &b, const void *src, size_t bytes) -> cudaError_t {
		cudaError_t e = b.ensure(bytes > 0 ? bytes : 16);
		if (e != cudaSuccess)
			return e;
		if (bytes > 0)
			return cudaMemcpy(b.p, src, bytes, cudaMemcpyHostToDevice);
		return cudaSuccess;
	};
	DeviceLayout4 lay4;
	flatten_bvh4(s->bvh, lay4);
	RNB_CUDA(up(s->d_nodes, lay.nodes.data(), lay.nodes.size() * sizeof(F4)));
	RNB_CUDA(up(s->d_nodes4, lay4.nodes.data(), lay4.nodes.size() * sizeof(F4)));
	RNB_CUDA(up(s->d_tris, lay.tris.data(), lay.tris.size() * sizeof(F4)));
	RNB_CUDA(up(s->d_ref_shade, ref.data(), ref.size() * sizeof(F4)));
	RNB_CUDA(up(s->d_phys_shade, phys.data(), phys.size() * sizeof(F4)));
	RNB_CUDA(up(s->d_emitters, em.data(), em.size() * sizeof(F4)));
	RNB_CUDA(s->d_status.ensure(256));
	RNB_CUDA(cudaMemset(s->d_status.p, 0, 256));

	SceneView v{};
	v.nodes = s->d_nodes.as<float4>();
	v.nodes4 = lay4.nodes.empty() ? nullptr : s->d_nodes4.as<float4>();
	v.root4_ref = lay4.root_ref;
	v.tris = s->d_tris.as<float4>();
	for (int a = 0; a < 3; a++) {
		v.root_lo[a] = lay.root_lo[a];
		v.root_hi[a] = lay.root_hi[a];
	}
	v.root_ref = lay.root_ref;
	v.n_tris = n;
	v.n_nodes = lay.internal_count;
	v.n_nodes4 = static_cast<int>(lay4.nodes.size() / 8);
	s->view = v;
	s->prepared = true;
	return RN_OK;
}

} // namespace rnb

rn_scene::~rn_scene() {
	if (stream)
		cudaStreamDestroy(stream);
}

using namespace rnb;

namespace {

// Fill defaults for the optional arrays and validate the vertices.
bool finish_triangle_set(TriangleSet &ts, std::string &err) {
	const size_t n = ts.size();
	for (float f : ts.v)
		if (!std::isfinite(f)) {
			err = "vertex coordinates must be finite";
			return false;
		}
	if (ts.rgb.size() != 3 * n)
		ts.rgb.assign(3 * n, 255);
	if (ts.ref_material.size() != n)
		ts.ref_material.assign(n, kRefDiffuse);
	if (ts.roughness.size() != n)
		ts.roughness.assign(n, 0.2f);
	if (ts.normal.size() != 3 * n) {
		ts.normal.resize(3 * n);
		for (size_t i = 0; i < n; i++) {
			Vec3 nn = loader_face_normal(&ts.v[9 * i]);
			ts.normal[3 * i] = nn.x;
			ts.normal[3 * i + 1] = nn.y;
			ts.normal[3 * i + 2] = nn.z;
		}
	}
	if (ts.vnormal.size() != 9 * n) { // every corner takes the face normal
		ts.vnormal.resize(9 * n);
		for (size_t i = 0; i < n; i++)
			for (int k = 0; k < 3; k++)
				for (int a = 0; a < 3; a++)
					ts.vnormal[9 * i + 3 * k + a] = ts.normal[3 * i + a];
	}
	if (ts.albedo.size() != 3 * n)
		ts.albedo.assign(3 * n, 0.8f);
	if (ts.emission.size() != 3 * n)
		ts.emission.assign(3 * n, 0.0f);
	if (ts.phys_material.size() != n)
		ts.phys_material.assign(n, kLambert);
	if (ts.phys_param.size() != n) {
		ts.phys_param.resize(n);
		for (size_t i = 0; i < n; i++)
			ts.phys_param[i] = ts.phys_material[i] == kDielectric ? 1.5f : 0.2f;
	}
	for (size_t i = 0; i < n; i++) {
		const int m = ts.ref_material[i];
		if (m < kRefDiffuse || m > kRefEmissive) {
			err = "reference material out of range";
			return false;
		}
		const int pm = ts.phys_material[i];
		if (pm < kLambert || pm > kDielectric) {
			err = "physical material out of range";
			return false;
		}
	}
	return true;
}

// Stage host arrays into the scene scratch buffer.
struct Staging {
	char *base = nullptr;
	size_t off = 0;
	template <typename T> T *take(size_t count) {
		size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
		T *p = reinterpret_cast<T *>(base + off);
		off += bytes;
		return p;
	}
};

rn_status check_status_word(int *d_err, cudaStream_t st, const char *what) {
	int h = 0;
	RNB_CUDA(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
	RNB_CUDA(cudaStreamSynchronize(st));
	if (h) {
		set_last_error(std::string(what) + ": traversal stack bound exceeded (corrupt scene)");
		return RN_ERR_INTERNAL;
	}
	return RN_OK;
}

} // namespace

extern "C" {

rn_scene *rn_scene_load_obj(const char *path, float scale) {
	TraceRange trace_range("rn_scene_load_obj");
	if (!path)
		return nullptr;
	try {
		rn_scene *s = new (std::nothrow) rn_scene();
		if (!s)
			return nullptr;
		std::string err;
		if (!load_obj(path, scale, s->tris, err) || !finish_triangle_set(s->tris, err)) {
			set_last_error(err);
			delete s;
			return nullptr;
		}
		return s;
	} catch (...) {
		set_last_error("exception while loading OBJ");
		return nullptr;
	}
}

void rn_scene_free(rn_scene *scene) { delete scene; }

int rn_scene_triangle_count(const rn_scene *scene) { return scene ? static_cast<int>(scene->tris.size()) : 0; }

const char *rn_version(void) { return "0.1.2"; }

const char *rn_pt_last_error(void) { return get_last_error(); }

rn_status rn_pt_scene_create(const rn_pt_scene_desc *desc, rn_scene **out) {
	if (!desc || !out || desc->num_triangles <= 0 || !desc->vertices) {
		set_last_error("rn_pt_scene_create: need a descriptor with vertices and num_triangles > 0");
		return RN_ERR_INVALID_ARGUMENT;
	}
	*out = nullptr;
	try {
		rn_scene *s = new (std::nothrow) rn_scene();
		if (!s)
			return RN_ERR_OUT_OF_MEMORY;
		const size_t n = static_cast<size_t>(desc->num_triangles);
		TriangleSet &ts = s->tris;
		ts.v.assign(desc->vertices, desc->vertices + 9 * n);
		if (desc->ref_rgb)
			ts.rgb.assign(desc->ref_rgb, desc->ref_rgb + 3 * n);
		if (desc->ref_material)
			ts.ref_material.assign(desc->ref_material, desc->ref_material + n);
		if (desc->ref_roughness)
			ts.roughness.assign(desc->ref_roughness, desc->ref_roughness + n);
		if (desc->ref_normal)
			ts.normal.assign(desc->ref_normal, desc->ref_normal + 3 * n);
		if (desc->ref_vertex_normals)
			ts.vnormal.assign(desc->ref_vertex_normals, desc->ref_vertex_normals + 9 * n);
		if (desc->albedo)
			ts.albedo.assign(desc->albedo, desc->albedo + 3 * n);
		if (desc->emission)
			ts.emission.assign(desc->emission, desc->emission + 3 * n);
		if (desc->material)
			ts.phys_material.assign(desc->material, desc->material + n);
		if (desc->material_param)
			ts.phys_param.assign(desc->material_param, desc->material_param + n);
		std::string err;
		if (!finish_triangle_set(ts, err)) {
			set_last_error("rn_pt_scene_create: " + err);
			delete s;
			return RN_ERR_INVALID_ARGUMENT;
		}
		*out = s;
		return RN_OK;
	} catch (const std::bad_alloc &) {
		set_last_error("rn_pt_scene_create: host allocation failed");
		return RN_ERR_OUT_OF_MEMORY;
	} catch (...) {
		set_last_error("rn_pt_scene_create: unexpected exception");
		return RN_ERR_INTERNAL;
	}
}

rn_status rn_pt_scene_prepare(rn_scene *scene) {
	TraceRange trace_range("rn_pt_scene_prepare");
	if (!scene) {
		set_last_error("rn_pt_scene_prepare: NULL scene");
		return RN_ERR_INVALID_ARGUMENT;
	}
	try {
		return prepare_scene(scene);
	} catch (const std::bad_alloc &) {
		set_last_error("host allocation failed while building the BVH");
		return RN_ERR_OUT_OF_MEMORY;
	} catch (...) {
		set_last_error("unexpected exception while preparing the scene");
		return RN_ERR_INTERNAL;
	}
}

rn_status rn_pt_scene_get_info(rn_scene *scene, rn_pt_scene_info *out) {
	if (!scene || !out) {
		set_last_error("rn_pt_scene_get_info: NULL argument");
		return RN_ERR_INVALID_ARGUMENT;
	}
	rn_status st = rn_pt_scene_prepare(scene);
	if (st != RN_OK)
		return st;
	out->num_triangles = static_cast<int>(scene->tris.size());
	out->internal_nodes = scene->internal_nodes;
	out->depth = scene->bvh.depth;
	out->device_bytes = static_cast<long long>(scene->d_nodes.bytes + scene->d_tris.bytes + scene->d_ref_shade.bytes +
	                                           scene->d_phys_shade.bytes + scene->d_emitters.bytes);
	out->build_ms = scene->build_ms;
	return RN_OK;
}

rn_status rn_pt_scene_get_triangles(const rn_scene *scene, float *vertices, int *ref_rgb, int *ref_material,
                                    float *ref_normal) {
	if (!scene) {
		set_last_error("rn_pt_scene_get_triangles: NULL scene");
		return RN_ERR_INVALID_ARGUMENT;
	}
	const TriangleSet &ts = scene->tris;
	if (vertices)
		std::memcpy(vertices, ts.v.data(), ts.v.size() * sizeof(float));
	if (ref_rgb)
		std::memcpy(ref_rgb, ts.rgb.data(), ts.rgb.size() * sizeof(int));
	if (ref_material)
		std::memcpy(ref_material, ts.ref_material.data(), ts.ref_material.size() * sizeof(int));
	if (ref_normal)
		std::memcpy(ref_normal, ts.normal.data(), ts.normal.size() * sizeof(float));
	return RN_OK;
}

rn_status rn_pt_scene_get_vertex_normals(const rn_scene *scene, float *vertex_normals) {
	if (!scene || !vertex_normals) {
		set_last_error("rn_pt_scene_get_vertex_normals: NULL argument");
		return RN_ERR_INVALID_ARGUMENT;
	}
	const TriangleSet &ts = scene->tris;
	std::memcpy(vertex_normals, ts.vnormal.data(), ts.vnormal.size() * sizeof(float));
	return RN_OK;
}

rn_status rn_pt_scene_dump_bvh(rn_scene *scene, int *order, int *node_count, float *bounds, int *links) {
	if (!scene || !node_count) {
		set_last_error("rn_pt_scene_dump_bvh: NULL argument");
		return RN_ERR_INVALID_ARGUMENT;
	}
	rn_status st;
	{
		std::lock_guard<std::mutex> lock(scene->mu);
		st = build_host(scene);
	}
	if (st != RN_OK)
		return st;
	const Bvh2 &b = scene->bvh;
	*node_count = static_cast<int>(b.nodes.size());
	if (order)
		std::memcpy(order, b.order.data(), b.order.size() * sizeof(int));
	for (size_t i = 0; i < b.nodes.size(); i++) {
		const BvhNode &nd = b.nodes[i];
		if (bounds) {
			const float bb[6] = {nd.bmin.x, nd.bmin.y, nd.bmin.z, nd.bmax.x, nd.bmax.y, nd.bmax.z};
			std::memcpy(bounds + 6 * i, bb, sizeof(bb));
		}
		if (links) {
			links[4 * i] = nd.left;
			links[4 * i + 1] = nd.right;
			links[4 * i + 2] = nd.start;
			links[4 * i + 3] = nd.count;
		}
	}
	return RN_OK;
}

rn_status rn_pt_scene_build_lbvh(rn_scene *scene, void *stream, double *build_ms) {
	TraceRange trace_range("rn_pt_scene_build_lbvh");
	if (!scene) {
		set_last_error("rn_pt_scene_build_lbvh: NULL scene");
		return RN_ERR_INVALID_ARGUMENT;
	}
	rn_status st = rn_pt_scene_prepare(scene);
	if (st != RN_OK)
		return st;
	cudaStream_t cs = pick_stream(scene, stream);
	std::lock_guard<std::mutex> lock(scene->scratch_mu);
	const int n = static_cast<int>(scene->tris.size());
	const auto t0 = std::chrono::steady_clock::now();
	const size_t vbytes = (scene->tris.v.size() * sizeof(float) + 255) & ~size_t(255);
	const size_t sbytes = lbvh_scratch_bytes(n);
	RNB_CUDA(scene->scratch.ensure(vbytes + sbytes));
	float *d_v9 = scene->scratch.as<float>();
	RNB_CUDA(cudaMemcpyAsync(d_v9, scene->tris.v.data(), scene->tris.v.size() * sizeof(float), cudaMemcpyHostToDevice,
	                         cs));
	scene->lbvh_ready = false; // the buffers below may move; the view is rebuilt on success
	RNB_CUDA(scene->d_lbvh_nodes.ensure(static_cast<size_t>(n > 1 ? n - 1 : 1) * 4 * sizeof(float4)));
	RNB_CUDA(scene->d_lbvh_tris.ensure(static_cast<size_t>(n) * 3 * sizeof(float4)));
	LbvhResult res{};
	RNB_CUDA(lbvh_build(d_v9, n, scene->scratch.as<char>() + vbytes, sbytes, scene->d_lbvh_nodes.as<float4>(),
	                    scene->d_lbvh_tris.as<float4>(), res, cs));
	if (res.depth > kStack - 2) {
		scene->lbvh_ready = false;
		set_last_error("rn_pt_scene_build_lbvh: the tree is deeper than the traversal stack (" +
		               std::to_string(res.depth) + " levels)");
		return RN_ERR_UNSUPPORTED;
	}
	SceneView v{};
	v.nodes = scene->d_lbvh_nodes.as<float4>();
	v.nodes4 = nullptr;
	v.tris = scene->d_lbvh_tris.as<float4>();
	for (int a = 0; a < 3; a++) {
		v.root_lo[a] = res.root_lo[a];
		v.root_hi[a] = res.root_hi[a];
	}
	v.root_ref = res.root_ref;
	v.root4_ref = 0;
	v.n_tris = n;
	v.n_nodes = n > 1 ? n - 1 : 0;
	v.n_nodes4 = 0;
	scene->lbvh_view = v;
	scene->lbvh_depth = res.depth;
	scene->lbvh_ready = true;
	if (build_ms)
		*build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
	return RN_OK;
}

// The tree a query runs on: the GPU-built one for RN_PT_LBVH (which implies
// nearest-first order), else the reference tree.
static rn_status query_view(rn_scene *scene, unsigned flags, const char *what, SceneView &view, int &order) {
	order = (flags & RN_PT_ORDER_NEAREST) ? kOrderNearest : kOrderReference;
	view = scene->view;
	if (flags & RN_PT_LBVH) {
		if (!scene->lbvh_ready) {
			set_last_error(std::string(what) + ": RN_PT_LBVH needs rn_pt_scene_build_lbvh first");
			return RN_ERR_INVALID_ARGUMENT;
		}
		view = scene->lbvh_view;
		order = kOrderNearest;
	}
	if (flags & RN_PT_WIDTH2)
		view.nodes4 = nullptr;
	return RN_OK;
}

rn_status rn_pt_trace_closest(rn_scene *scene, int n, const float *origins, const float *directions, const int *ignore,
                              unsigned flags, void *stream, int *tri, float *t, float *u, float *v) {
	TraceRange trace_range("rn_pt_trace_closest");
	if (!scene || n < 0 || (n > 0 && (!origins || !directions || !tri))) {
		set_last_error("rn_pt_trace_closest: invalid argument");
		return RN_ERR_INVALID_ARGUMENT;
	}
	rn_status st = rn_pt_scene_prepare(scene);
	if (st != RN_OK || n == 0)
		return st;
	int order = kOrderReference;
	SceneView view;
	st = query_view(scene, flags, "rn_pt_trace_closest", view, order);
	if (st != RN_OK)
		return st;
	cudaStream_t cs = pick_stream(scene, stream);
	std::lock_guard<std::mutex> lock(scene->scratch_mu);
	const size_t nn = static_cast<size_t>(n);
	RNB_CUDA(scene->scratch.ensure(nn * 4 * 13 + 256 * 12));
	Staging sg{scene->scratch.as<char>()};
	int *d_err = sg.take<int>(1);
	RNB_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), cs));
	if (flags & RN_PT_DEVICE_POINTERS) {
		RNB_CUDA(launch_trace_closest(view, n, origins, directions, ignore, order, tri, t, u, v,
		                              scene->d_status.as<int>(), cs));
		return RN_OK;
	}
	float *d_o = sg.take<float>(3 * nn), *d_d = sg.take<float>(3 * nn);
	int *d_ig = ignore ? sg.take<int>(nn) : nullptr;
	int *d_tri = sg.take<int>(nn);
	float *d_t = sg.take<float>(nn), *d_u = sg.take<float>(nn), *d_v = sg.take<float>(nn);
	RNB_CUDA(cudaMemcpyAsync(d_o, origins, 12 * nn, cudaMemcpyHostToDevice, cs));
	RNB_CUDA(cudaMemcpyAsync(d_d, directions, 12 * nn, cudaMemcpyHostToDevice, cs));
	if (d_ig)
		RNB_CUDA(cudaMemcpyAsync(d_ig, ignore, 4 * nn, cudaMemcpyHostToDevice, cs));
	RNB_CUDA(launch_trace_closest(view, n, d_o, d_d, d_ig, order, d_tri, d_t, d_u, d_v, d_err, cs));
	RNB_CUDA(cudaMemcpyAsync(tri, d_tri, 4 * nn, cudaMemcpyDeviceToHost, cs));
	if (t)
		RNB_CUDA(cudaMemcpyAsync(t, d_t, 4 * nn, cudaMemcpyDeviceToHost, cs));
	if (u)
		RNB_CUDA(cudaMemcpyAsync(u, d_u, 4 * nn, cudaMemcpyDeviceToHost, cs));
	if (v)
		RNB_CUDA(cudaMemcpyAsync(v, d_v, 4 * nn, cudaMemcpyDeviceToHost, cs));
	return check_status_word(d_err, cs, "rn_pt_trace_closest");
}

rn_status rn_pt_trace_any(rn_scene *scene, int n, const float *origins, const float *directions, const float *tmax,
                          const int *ignore, unsigned flags, void *stream, int *occluded) {
	TraceRange trace_range("rn_pt_trace_any");
	if (!scene || n < 0 || (n > 0 && (!origins || !directions || !tmax || !occluded))) {
		set_last_error("rn_pt_trace_any: invalid argument");
		return RN_ERR_INVALID_ARGUMENT;
	}
	rn_status st = rn_pt_scene_prepare(scene);
	if (st != RN_OK || n == 0)
		return st;
	int order = kOrderReference;
	SceneView view;
	st = query_view(scene, flags, "rn_pt_trace_any", view, order);
	if (st != RN_OK)
		return st;
	cudaStream_t cs = pick_stream(scene, stream);
	std::lock_guard<std::mutex> lock(scene->scratch_mu);
	const size_t nn = static_cast<size_t>(n);
	RNB_CUDA(scene->scratch.ensure(nn * 4 * 10 + 256 * 8));
	Staging sg{scene->scratch.as<char>()};
	int *d_err = sg.take<int>(1);
	RNB_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), cs));
	if (flags & RN_PT_DEVICE_POINTERS) {
		RNB_CUDA(launch_trace_any(view, n, origins, directions, tmax, ignore, occluded,
		                          scene->d_status.as<int>(), cs));
		return RN_OK;
	}
	float *d_o = sg.take<float>(3 * nn), *d_d = sg.take<float>(3 * nn), *d_tm = sg.take<float>(nn);
	int *d_ig = ignore ? sg.take<int>(nn) : nullptr;
	int *d_occ = sg.take<int>(nn);
	RNB_CUDA(cudaMemcpyAsync(d_o, origins, 12 * nn, cudaMemcpyHostToDevice, cs));
	RNB_CUDA(cudaMemcpyAsync(d_d, directions, 12 * nn, cudaMemcpyHostToDevice, cs));
	RNB_CUDA(cudaMemcpyAsync(d_tm, tmax, 4 * nn, cudaMemcpyHostToDevice, cs));
	if (d_ig)
		RNB_CUDA(cudaMemcpyAsync(d_ig, ignore, 4 * nn, cudaMemcpyHostToDevice, cs));
	RNB_CUDA(launch_trace_any(view, n, d_o, d_d, d_tm, d_ig, d_occ, d_err, cs));
	RNB_CUDA(cudaMemcpyAsync(occluded, d_occ, 4 * nn, cudaMemcpyDeviceToHost, cs));
	return check_status_word(d_err, cs, "rn_pt_trace_any");
}

} // extern "C"

rn_status rn_pt_inject_allocation_failure(long long after) {
	g_alloc_countdown.store(after < 0 ? -1 : after);
	return RN_OK;
}
