// Drop-in rn_render / rn_save_png and the reference-mode entry point.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gi.hpp"
#include "photon.hpp"
#include "refmode.hpp"
#include "scene_impl.hpp"
#include "trace_range.hpp"

using namespace rnb;

namespace {

// Camera::lookAt (src/Camera.cpp:27-33) with glm's normalize / cross order.
void look_at(const float pos[3], const float target[3], float orient[9]) {
	auto normalize = [](float v[3]) {
		const float d = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
		const float s = 1.0f / std::sqrt(d);
		v[0] *= s;
		v[1] *= s;
		v[2] *= s;
	};
	auto cross = [](const float x[3], const float y[3], float o[3]) {
		o[0] = x[1] * y[2] - y[1] * x[2];
		o[1] = x[2] * y[0] - y[2] * x[0];
		o[2] = x[0] * y[1] - y[0] * x[1];
	};
	float fwd[3] = {pos[0] - target[0], pos[1] - target[1], pos[2] - target[2]};
	normalize(fwd);
	const float world_up[3] = {0.0f, 1.0f, 0.0f};
	float right[3], up[3];
	cross(world_up, fwd, right);
	normalize(right);
	cross(fwd, right, up);
	std::memcpy(orient, right, 12);
	std::memcpy(orient + 3, up, 12);
	std::memcpy(orient + 6, fwd, 12);
}

RefLight to_ref_light(const rn_light &l) {
	RefLight r;
	r.type = l.type;
	std::memcpy(r.position, l.position, 12);
	std::memcpy(r.direction, l.direction, 12);
	std::memcpy(r.colour, l.colour, 12);
	r.intensity = l.intensity;
	r.radius = l.radius;
	r.cone_cos = l.cone_cos;
	r.atten_constant = l.atten_constant;
	r.atten_linear = l.atten_linear;
	r.atten_quadratic = l.atten_quadratic;
	std::memcpy(r.u_axis, l.u_axis, 12);
	std::memcpy(r.v_axis, l.v_axis, 12);
	return r;
}

// The reference's default Light with radius 0.15 (src/Light.h:13-29, src/Renderer.cpp:1129-1134).
RefLight default_light() {
	RefLight r{};
	r.type = kLightPoint;
	r.position[0] = 0.0f;
	r.position[1] = 0.95f;
	r.position[2] = 0.0f;
	r.direction[1] = -1.0f;
	r.colour[0] = r.colour[1] = r.colour[2] = 1.0f;
	r.intensity = 40.0f;
	r.radius = 0.15f;
	r.cone_cos = 0.9f;
	r.atten_quadratic = 12.566370f;
	r.u_axis[0] = 0.3f;
	r.v_axis[2] = 0.3f;
	return r;
}

// --- minimal PNG writer: 8-bit RGBA, zlib stored (uncompressed) blocks ---
uint32_t crc_table[256];
bool crc_ready = false;
uint32_t crc32(const unsigned char *p, size_t n, uint32_t c = 0xffffffffu) {
	if (!crc_ready) {
		for (uint32_t i = 0; i < 256; i++) {
			uint32_t k = i;
			for (int j = 0; j < 8; j++)
				k = (k & 1) ? 0xedb88320u ^ (k >> 1) : (k >> 1);
			crc_table[i] = k;
		}
		crc_ready = true;
	}
	for (size_t i = 0; i < n; i++)
		c = crc_table[(c ^ p[i]) & 0xff] ^ (c >> 8);
	return c;
}
void put32(std::vector<unsigned char> &v, uint32_t x) {
	v.push_back(static_cast<unsigned char>(x >> 24));
	v.push_back(static_cast<unsigned char>(x >> 16));
	v.push_back(static_cast<unsigned char>(x >> 8));
	v.push_back(static_cast<unsigned char>(x));
}
void chunk(std::vector<unsigned char> &out, const char *type, const std::vector<unsigned char> &data) {
	put32(out, static_cast<uint32_t>(data.size()));
	std::vector<unsigned char> td(type, type + 4);
	td.insert(td.end(), data.begin(), data.end());
	out.insert(out.end(), td.begin(), td.end());
	put32(out, crc32(td.data(), td.size()) ^ 0xffffffffu);
}

} // namespace

extern "C" {

void rn_pt_ref_params_init(rn_pt_ref_params *p, int width, int height, float cam_z, int samples) {
	if (!p)
		return;
	std::memset(p, 0, sizeof(*p));
	p->width = width;
	p->height = height;
	p->position[2] = cam_z;
	p->focal_length = 2.0f;
	p->scale = 150.0f;
	p->ortho_scale = 1.0f;
	p->samples = samples;
	p->max_depth = 4;
	p->focus_distance = 4.0f;
}

rn_status rn_pt_render_reference(rn_scene *scene, const rn_pt_ref_params *prm, unsigned flags, void *stream,
                                 uint32_t *argb, float *mean_rgb) {
	TraceRange trace_range("rn_pt_render_reference");
	if (!scene || !prm || prm->width <= 0 || prm->height <= 0 || (!argb && !mean_rgb)) {
		set_last_error("rn_pt_render_reference: invalid argument");
		return RN_ERR_INVALID_ARGUMENT;
	}
	if (prm->num_lights < 0 || prm->num_lights > kMaxRefLights || (prm->num_lights > 0 && !prm->lights)) {
		set_last_error("rn_pt_render_reference: num_lights must be in [0, 16] with a lights array");
		return RN_ERR_INVALID_ARGUMENT;
	}
	if (prm->max_depth < 0 || prm->max_depth > kMaxRefDepth) {
		set_last_error("rn_pt_render_reference: max_depth must be in [0, 15]");
		return RN_ERR_INVALID_ARGUMENT;
	}
	const long npix = static_cast<long>(prm->width) * prm->height;
	if (npix > (1L << 28)) {
		set_last_error("rn_pt_render_reference: image too large");
		return RN_ERR_INVALID_ARGUMENT;
	}
	rn_status st = rn_pt_scene_prepare(scene);
	if (st != RN_OK)
		return st;
	RefParams p{};
	p.width = prm->width;
	p.height = prm->height;
	std::memcpy(p.position, prm->position, 12);
	look_at(prm->position, prm->target, p.orient);
	p.f = prm->focal_length * prm->scale;
	p.orthographic = prm->orthographic;
	p.ortho_scale = prm->ortho_scale;
	p.samples = prm->samples;
	p.max_depth = prm->max_depth;
	if (prm->num_lights == 0) {
		p.num_lights = 1;
		p.lights[0] = default_light();
	} else {
		p.num_lights = prm->num_lights;
		for (int i = 0; i < prm->num_lights; i++)
			p.lights[i] = to_ref_light(prm->lights[i]);
	}
	p.aperture = prm->aperture;
	p.focus_distance = prm->focus_distance;
	std::memcpy(p.camera_motion, prm->camera_motion, 12);
	p.aperture_blades = prm->aperture_blades;
	p.aperture_args_right_to_left = 1;

	cudaStream_t cs = pick_stream(scene, stream);
	std::lock_guard<std::mutex> lock(scene->scratch_mu);
	// Path records and shadow-ray results: the whole frame when it fits in 2 GiB,
	// else pixel chunks.
	const size_t per_pixel = ref_defer_bytes_per_pixel(p);
	const size_t defer =
	    kRefDeferFixedBytes + std::min(static_cast<size_t>(npix) * per_pixel, std::max(size_t(2) << 30, per_pixel));
	const size_t head = 256 + ((sizeof(RefParams) + 255) & ~size_t(255)) + ((static_cast<size_t>(npix) * 4 + 255) &
	                    ~size_t(255)) + ((static_cast<size_t>(npix) * 12 + 255) & ~size_t(255));
	RNB_CUDA(scene->scratch.ensure(head + defer));
	char *base = scene->scratch.as<char>();
	int *d_err = reinterpret_cast<int *>(base);
	RefParams *d_p = reinterpret_cast<RefParams *>(base + 256);
	char *rest = base + 256 + ((sizeof(RefParams) + 255) & ~size_t(255));
	uint32_t *d_argb = reinterpret_cast<uint32_t *>(rest);
	float *d_mean = reinterpret_cast<float *>(rest + ((static_cast<size_t>(npix) * 4 + 255) & ~size_t(255)));
	const bool dev = (flags & RN_PT_DEVICE_POINTERS) != 0;
	RNB_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), cs));
	RNB_CUDA(cudaMemcpyAsync(d_p, &p, sizeof(p), cudaMemcpyHostToDevice, cs));
	uint32_t *o_argb = argb ? (dev ? argb : d_argb) : d_argb;
	float *o_mean = mean_rgb ? (dev ? mean_rgb : d_mean) : nullptr;
	RNB_CUDA(launch_render_reference(scene->view, scene->d_ref_shade.as<float4>(), p, d_p, o_argb, o_mean, d_err,
	                                 base + head, defer, cs));
	if (!dev) {
		if (argb)
			RNB_CUDA(cudaMemcpyAsync(argb, d_argb, static_cast<size_t>(npix) * 4, cudaMemcpyDeviceToHost, cs));
		if (mean_rgb)
			RNB_CUDA(cudaMemcpyAsync(mean_rgb, d_mean, static_cast<size_t>(npix) * 12, cudaMemcpyDeviceToHost, cs));
	}
	// The parameter block lives in scratch: finish before releasing the lock.
	int h = 0;
	RNB_CUDA(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, cs));
	RNB_CUDA(cudaStreamSynchronize(cs));
	if (h) {
		set_last_error("rn_pt_render_reference: traversal stack bound exceeded (corrupt scene)");
		return RN_ERR_INTERNAL;
	}
	return RN_OK;
}

rn_status rn_pt_render_raytraced(rn_scene *scene, const rn_pt_ref_params *prm, int shading, float fog_density,
                                 const float *fog_colour, unsigned flags, void *stream, uint32_t *argb) {
	TraceRange trace_range("rn_pt_render_raytraced");
	if (!scene || !prm || prm->width <= 0 || prm->height <= 0 || !argb) {
		set_last_error("rn_pt_render_raytraced: invalid argument");
		return RN_ERR_INVALID_ARGUMENT;
	}
	if (shading < 0 || shading > 2) {
		set_last_error("rn_pt_render_raytraced: shading must be RN_PT_SHADING_FLAT, _GOURAUD or _PHONG");
		return RN_ERR_INVALID_ARGUMENT;
	}
	if (prm->num_lights < 0 || prm->num_lights > kMaxRefLights || (prm->num_lights > 0 && !prm->lights)) {
		set_last_error("rn_pt_render_raytraced: num_lights must be in [0, 16] with a lights array");
		return RN_ERR_INVALID_ARGUMENT;
	}
	if (prm->max_depth < 0 || prm->max_depth > kMaxWhittedDepth) {
		set_last_error("rn_pt_render_raytraced: max_depth must be in [0, 8]");
		return RN_ERR_INVALID_ARGUMENT;
	}
	const long npix = static_cast<long>(prm->width) * prm->height;
	if (npix > (1L << 28)) {
		set_last_error("rn_pt_render_raytraced: image too large");
		return RN_ERR_INVALID_ARGUMENT;
	}
	rn_status st = rn_pt_scene_prepare(scene);
	if (st != RN_OK)
		return st;
	cudaStream_t cs = pick_stream(scene, stream);
	{
		// Vertices and vertex normals in the caller's triangle order, 6 float4 each.
		std::lock_guard<std::mutex> lock(scene->mu);
		if (!scene->ref_geom_ready) {
			const TriangleSet &ts = scene->tris;
			const size_t n = ts.size();
			std::vector<float4> g(6 * n);
			for (size_t i = 0; i < n; i++)
				for (int k = 0; k < 3; k++) {
					g[6 * i + k] = make_float4(ts.v[9 * i + 3 * k], ts.v[9 * i + 3 * k + 1], ts.v[9 * i + 3 * k + 2], 0.0f);
					g[6 * i + 3 + k] = make_float4(ts.vnormal[9 * i + 3 * k], ts.vnormal[9 * i + 3 * k + 1],
					                               ts.vnormal[9 * i + 3 * k + 2], 0.0f);
				}
			RNB_CUDA(scene->d_ref_geom.ensure(g.size() * sizeof(float4)));
			RNB_CUDA(cudaMemcpy(scene->d_ref_geom.p, g.data(), g.size() * sizeof(float4), cudaMemcpyHostToDevice));
			scene->ref_geom_ready = true;
		}
	}
	RefParams p{};
	p.width = prm->width;
	p.height = prm->height;
	std::memcpy(p.position, prm->position, 12);
	look_at(prm->position, prm->target, p.orient);
	p.f = prm->focal_length * prm->scale;
	p.orthographic = prm->orthographic;
	p.ortho_scale = prm->ortho_scale;
	p.max_depth = prm->max_depth;
	if (prm->num_lights == 0) {
		p.num_lights = 1;
		p.lights[0] = default_light();
	} else {
		p.num_lights = prm->num_lights;
		for (int i = 0; i < prm->num_lights; i++)
			p.lights[i] = to_ref_light(prm->lights[i]);
	}
	p.shading = shading;
	p.fog_density = fog_density;
	const float fog_default[3] = {200.0f, 210.0f, 230.0f};
	std::memcpy(p.fog_colour, fog_colour ? fog_colour : fog_default, 12);

	std::lock_guard<std::mutex> lock(scene->scratch_mu);
	const size_t pb = (sizeof(RefParams) + 255) & ~size_t(255);
	RNB_CUDA(scene->scratch.ensure(256 + pb + static_cast<size_t>(npix) * 4 + 256));
	char *base = scene->scratch.as<char>();
	int *d_err = reinterpret_cast<int *>(base);
	RefParams *d_p = reinterpret_cast<RefParams *>(base + 256);
	uint32_t *d_argb = reinterpret_cast<uint32_t *>(base + 256 + pb);
	const bool dev = (flags & RN_PT_DEVICE_POINTERS) != 0;
	RNB_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), cs));
	RNB_CUDA(cudaMemcpyAsync(d_p, &p, sizeof(p), cudaMemcpyHostToDevice, cs));
	RNB_CUDA(launch_render_raytraced(scene->view, scene->d_ref_shade.as<float4>(), scene->d_ref_geom.as<float4>(), d_p,
	                                 p.width, p.height, dev ? argb : d_argb, d_err, cs));
	if (!dev)
		RNB_CUDA(cudaMemcpyAsync(argb, d_argb, static_cast<size_t>(npix) * 4, cudaMemcpyDeviceToHost, cs));
	// The parameter block lives in scratch: finish before releasing the lock.
	int h = 0;
	RNB_CUDA(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, cs));
	RNB_CUDA(cudaStreamSynchronize(cs));
	if (h) {
		set_last_error("rn_pt_render_raytraced: traversal stack bound exceeded (corrupt scene)");
		return RN_ERR_INTERNAL;
	}
	return RN_OK;
}

rn_status rn_pt_render_photon_mapped(rn_scene *scene, const rn_pt_ref_params *prm, int num_photons, int gather_rays,
                                     unsigned flags, void *stream, uint32_t *argb, unsigned *num_stored) {
	TraceRange trace_range("rn_pt_render_photon_mapped");
	if (!scene || !prm || prm->width <= 0 || prm->height <= 0 || !argb) {
		set_last_error("rn_pt_render_photon_mapped: invalid argument");
		return RN_ERR_INVALID_ARGUMENT;
	}
	if (num_photons < 1 || num_photons > kMaxPhotons || gather_rays < 0 || gather_rays > 4096) {
		set_last_error("rn_pt_render_photon_mapped: need 1 <= num_photons <= 4194304 and 0 <= gather_rays <= 4096");
		return RN_ERR_INVALID_ARGUMENT;
	}
	if (prm->num_lights < 0 || prm->num_lights > kMaxRefLights || (prm->num_lights > 0 && !prm->lights)) {
		set_last_error("rn_pt_render_photon_mapped: num_lights must be in [0, 16] with a lights array");
		return RN_ERR_INVALID_ARGUMENT;
	}
	const long npix = static_cast<long>(prm->width) * prm->height;
	if (npix > (1L << 28)) {
		set_last_error("rn_pt_render_photon_mapped: image too large");
		return RN_ERR_INVALID_ARGUMENT;
	}
	rn_status st = rn_pt_scene_prepare(scene);
	if (st != RN_OK)
		return st;
	RefParams p{};
	p.width = prm->width;
	p.height = prm->height;
	std::memcpy(p.position, prm->position, 12);
	look_at(prm->position, prm->target, p.orient);
	p.f = prm->focal_length * prm->scale;
	if (prm->num_lights == 0) {
		p.num_lights = 1;
		p.lights[0] = default_light();
	} else {
		p.num_lights = prm->num_lights;
		for (int i = 0; i < prm->num_lights; i++)
			p.lights[i] = to_ref_light(prm->lights[i]);
	}
	size_t map_bytes = 0;
	RNB_CUDA(photon_scratch_bytes(num_photons, map_bytes));
	cudaStream_t cs = pick_stream(scene, stream);
	std::lock_guard<std::mutex> lock(scene->scratch_mu);
	const size_t pb = (sizeof(RefParams) + 255) & ~size_t(255);
	const size_t img = (static_cast<size_t>(npix) * 4 + 255) & ~size_t(255);
	RNB_CUDA(scene->scratch.ensure(256 + pb + img + map_bytes));
	char *base = scene->scratch.as<char>();
	int *d_err = reinterpret_cast<int *>(base);
	RefParams *d_p = reinterpret_cast<RefParams *>(base + 256);
	uint32_t *d_argb = reinterpret_cast<uint32_t *>(base + 256 + pb);
	void *d_map = base + 256 + pb + img;
	const bool dev = (flags & RN_PT_DEVICE_POINTERS) != 0;
	RNB_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), cs));
	RNB_CUDA(cudaMemcpyAsync(d_p, &p, sizeof(p), cudaMemcpyHostToDevice, cs));
	unsigned stored = 0;
	RNB_CUDA(launch_photon_mapped(scene->view, scene->d_ref_shade.as<float4>(), p, d_p, num_photons, gather_rays, d_map,
	                              map_bytes, dev ? argb : d_argb, d_err, cs, &stored));
	if (num_stored)
		*num_stored = stored;
	if (!dev)
		RNB_CUDA(cudaMemcpyAsync(argb, d_argb, static_cast<size_t>(npix) * 4, cudaMemcpyDeviceToHost, cs));
	int h = 0;
	RNB_CUDA(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, cs));
	RNB_CUDA(cudaStreamSynchronize(cs));
	if (h) {
		set_last_error("rn_pt_render_photon_mapped: traversal stack bound exceeded (corrupt scene)");
		return RN_ERR_INTERNAL;
	}
	return RN_OK;
}

namespace {

// Validation and the camera shared by the bidirectional and Metropolis renderers.
rn_status gi_params(const char *fn, rn_scene *scene, const rn_pt_ref_params *prm, float exposure, GiParams &p) {
	if (!scene || !prm || prm->width <= 0 || prm->height <= 0 || !std::isfinite(exposure)) {
		set_last_error(std::string(fn) + ": invalid argument");
		return RN_ERR_INVALID_ARGUMENT;
	}
	if (static_cast<long>(prm->width) * prm->height > (1L << 26)) {
		set_last_error(std::string(fn) + ": image too large");
		return RN_ERR_INVALID_ARGUMENT;
	}
	p = GiParams{};
	p.width = prm->width;
	p.height = prm->height;
	std::memcpy(p.position, prm->position, 12);
	look_at(prm->position, prm->target, p.orient);
	p.f = prm->focal_length * prm->scale;
	p.exposure = exposure;
	return rn_pt_scene_prepare(scene);
}

} // namespace

rn_status rn_pt_render_bidirectional(rn_scene *scene, const rn_pt_ref_params *prm, int samples, float exposure, int rng,
                                     unsigned long long seed, unsigned flags, void *stream, uint32_t *argb,
                                     float *rgb) {
	TraceRange trace_range("rn_pt_render_bidirectional");
	GiParams p;
	rn_status st = gi_params("rn_pt_render_bidirectional", scene, prm, exposure, p);
	if (st != RN_OK)
		return st;
	if (!argb || samples < 1 || samples > (1 << 16) || (rng != RN_PT_RNG_REFERENCE && rng != RN_PT_RNG_COUNTER)) {
		set_last_error("rn_pt_render_bidirectional: need argb, 1 <= samples <= 65536 and a known rng");
		return RN_ERR_INVALID_ARGUMENT;
	}
	p.samples = samples;
	p.seed = seed;
	const bool ref_stream = rng == RN_PT_RNG_REFERENCE;
	const size_t budget = size_t(512) << 20;
	const long npix = static_cast<long>(p.width) * p.height;
	const bool dev = (flags & RN_PT_DEVICE_POINTERS) != 0;
	cudaStream_t cs = pick_stream(scene, stream);
	std::lock_guard<std::mutex> lock(scene->scratch_mu);
	const size_t img = dev ? 0 : ((static_cast<size_t>(npix) * 4 + 255) & ~size_t(255));
	const size_t frgb = (dev || !rgb) ? 0 : ((static_cast<size_t>(npix) * 12 + 255) & ~size_t(255));
	RNB_CUDA(scene->scratch.ensure(256 + img + frgb + bdpt_scratch_bytes(p, ref_stream, budget)));
	char *base = scene->scratch.as<char>();
	int *d_err = reinterpret_cast<int *>(base);
	uint32_t *d_argb = dev ? argb : reinterpret_cast<uint32_t *>(base + 256);
	float *d_rgb = dev ? rgb : (rgb ? reinterpret_cast<float *>(base + 256 + img) : nullptr);
	RNB_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), cs));
	RNB_CUDA(launch_bdpt(scene->view, scene->d_ref_shade.as<float4>(), p, ref_stream, budget, base + 256 + img + frgb,
	                     d_argb, d_rgb, d_err, cs));
	if (!dev) {
		RNB_CUDA(cudaMemcpyAsync(argb, d_argb, static_cast<size_t>(npix) * 4, cudaMemcpyDeviceToHost, cs));
		if (rgb)
			RNB_CUDA(cudaMemcpyAsync(rgb, d_rgb, static_cast<size_t>(npix) * 12, cudaMemcpyDeviceToHost, cs));
	}
	int h = 0;
	RNB_CUDA(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, cs));
	RNB_CUDA(cudaStreamSynchronize(cs));
	if (h) {
		set_last_error("rn_pt_render_bidirectional: traversal stack bound exceeded (corrupt scene)");
		return RN_ERR_INTERNAL;
	}
	return RN_OK;
}

rn_status rn_pt_render_metropolis(rn_scene *scene, const rn_pt_ref_params *prm, long long mutations, float exposure,
                                  int chains, int bootstrap, unsigned long long seed, unsigned flags, void *stream,
                                  uint32_t *argb, float *rgb, double *mean_luminance) {
	TraceRange trace_range("rn_pt_render_metropolis");
	GiParams p;
	rn_status st = gi_params("rn_pt_render_metropolis", scene, prm, exposure, p);
	if (st != RN_OK)
		return st;
	if (!argb || mutations < 1 || mutations > (1LL << 40) || chains < 0 || chains > (1 << 22) || bootstrap < 1 ||
	    bootstrap > kMltMaxBootstrap) {
		set_last_error("rn_pt_render_metropolis: need argb, 1 <= mutations <= 2^40, 0 <= chains <= 2^22 and "
		               "1 <= bootstrap <= 2^24");
		return RN_ERR_INVALID_ARGUMENT;
	}
	if (chains == 0)
		chains = static_cast<int>(std::max<long long>(1, std::min<long long>(mutations / 16, 1 << 21)));
	if (chains > mutations || mutations / chains >= (1LL << 32)) {
		set_last_error("rn_pt_render_metropolis: need chains <= mutations and mutations / chains < 2^32");
		return RN_ERR_INVALID_ARGUMENT;
	}
	p.mutations = mutations;
	p.chains = chains;
	p.bootstrap = bootstrap;
	p.seed = seed;
	const long npix = static_cast<long>(p.width) * p.height;
	const bool dev = (flags & RN_PT_DEVICE_POINTERS) != 0;
	cudaStream_t cs = pick_stream(scene, stream);
	std::lock_guard<std::mutex> lock(scene->scratch_mu);
	const size_t img = dev ? 0 : ((static_cast<size_t>(npix) * 4 + 255) & ~size_t(255));
	const size_t frgb = (dev || !rgb) ? 0 : ((static_cast<size_t>(npix) * 12 + 255) & ~size_t(255));
	RNB_CUDA(scene->scratch.ensure(256 + img + frgb + mlt_scratch_bytes(p)));
	char *base = scene->scratch.as<char>();
	int *d_err = reinterpret_cast<int *>(base);
	double *d_b = reinterpret_cast<double *>(base + 8);
	uint32_t *d_argb = dev ? argb : reinterpret_cast<uint32_t *>(base + 256);
	float *d_rgb = dev ? rgb : (rgb ? reinterpret_cast<float *>(base + 256 + img) : nullptr);
	RNB_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), cs));
	RNB_CUDA(launch_mlt(scene->view, scene->d_ref_shade.as<float4>(), p, base + 256 + img + frgb, d_argb, d_rgb,
	                    dev && mean_luminance ? mean_luminance : d_b, d_err, cs));
	if (!dev) {
		RNB_CUDA(cudaMemcpyAsync(argb, d_argb, static_cast<size_t>(npix) * 4, cudaMemcpyDeviceToHost, cs));
		if (rgb)
			RNB_CUDA(cudaMemcpyAsync(rgb, d_rgb, static_cast<size_t>(npix) * 12, cudaMemcpyDeviceToHost, cs));
		if (mean_luminance)
			RNB_CUDA(cudaMemcpyAsync(mean_luminance, d_b, sizeof(double), cudaMemcpyDeviceToHost, cs));
	}
	int h = 0;
	RNB_CUDA(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, cs));
	RNB_CUDA(cudaStreamSynchronize(cs));
	if (h) {
		set_last_error("rn_pt_render_metropolis: traversal stack bound exceeded (corrupt scene)");
		return RN_ERR_INTERNAL;
	}
	return RN_OK;
}

int rn_render(const rn_scene *scene, rn_render_mode mode, int width, int height, float cam_z, int samples,
              unsigned char *rgba) {
	TraceRange trace_range("rn_render");
	if (!scene || !rgba || width <= 0 || height <= 0)
		return 0;
	if (mode != RN_PATHTRACED && mode != RN_RAYTRACED) {
		set_last_error("rn_render: RN_PATHTRACED and RN_RAYTRACED are served by rednoise-b200");
		return 0;
	}
	try {
		rn_pt_ref_params p;
		rn_pt_ref_params_init(&p, width, height, cam_z, samples);
		std::vector<uint32_t> canvas(static_cast<size_t>(width) * height);
		// The C ABI takes a const scene; preparation only fills lazily built caches.
		// renderRaytraced's defaults: Phong shading, depth 4, no fog (src/Renderer.h:43-46).
		rn_status st = mode == RN_RAYTRACED
		                   ? rn_pt_render_raytraced(const_cast<rn_scene *>(scene), &p, RN_PT_SHADING_PHONG, 0.0f,
		                                            nullptr, 0, nullptr, canvas.data())
		                   : rn_pt_render_reference(const_cast<rn_scene *>(scene), &p, 0, nullptr, canvas.data(),
		                                            nullptr);
		if (st != RN_OK)
			return 0;
		// Canvas 0xAARRGGBB -> RGBA8 (src/capi.cpp:70-78).
		for (size_t i = 0; i < canvas.size(); i++) {
			const uint32_t px = canvas[i];
			rgba[4 * i + 0] = static_cast<unsigned char>((px >> 16) & 0xFF);
			rgba[4 * i + 1] = static_cast<unsigned char>((px >> 8) & 0xFF);
			rgba[4 * i + 2] = static_cast<unsigned char>(px & 0xFF);
			rgba[4 * i + 3] = static_cast<unsigned char>((px >> 24) & 0xFF);
		}
		return 1;
	} catch (...) {
		set_last_error("rn_render: unexpected exception");
		return 0;
	}
}

int rn_save_png(const char *path, int width, int height, const unsigned char *rgba) {
	if (!path || !rgba || width <= 0 || height <= 0)
		return 0;
	try {
		// Raw scanlines, filter byte 0, wrapped in stored deflate blocks.
		const size_t row = static_cast<size_t>(width) * 4;
		std::vector<unsigned char> raw;
		raw.reserve((row + 1) * static_cast<size_t>(height));
		for (int y = 0; y < height; y++) {
			raw.push_back(0);
			raw.insert(raw.end(), rgba + row * y, rgba + row * (y + 1));
		}
		std::vector<unsigned char> z = {0x78, 0x01};
		size_t off = 0;
		do {
			const size_t n = std::min<size_t>(65535, raw.size() - off);
			const bool last = off + n == raw.size();
			z.push_back(last ? 1 : 0);
			z.push_back(static_cast<unsigned char>(n & 0xff));
			z.push_back(static_cast<unsigned char>(n >> 8));
			z.push_back(static_cast<unsigned char>(~n & 0xff));
			z.push_back(static_cast<unsigned char>((~n >> 8) & 0xff));
			z.insert(z.end(), raw.begin() + static_cast<long>(off), raw.begin() + static_cast<long>(off + n));
			off += n;
		} while (off < raw.size());
		uint32_t a = 1, b = 0;
		for (unsigned char c : raw) {
			a = (a + c) % 65521u;
			b = (b + a) % 65521u;
		}
		put32(z, (b << 16) | a);
		std::vector<unsigned char> out = {0x89, 'P', 'N', 'G', 0x0d, 0x0a, 0x1a, 0x0a};
		std::vector<unsigned char> ihdr;
		put32(ihdr, static_cast<uint32_t>(width));
		put32(ihdr, static_cast<uint32_t>(height));
		ihdr.insert(ihdr.end(), {8, 6, 0, 0, 0});
		chunk(out, "IHDR", ihdr);
		chunk(out, "IDAT", z);
		chunk(out, "IEND", {});
		FILE *f = std::fopen(path, "wb");
		if (!f)
			return 0;
		const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
		return (std::fclose(f) == 0 && ok) ? 1 : 0;
	} catch (...) {
		return 0;
	}
}

} // extern "C"
