// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// A flat extern "C" shim over the reference renderer's C++ engine, compiled
// together with the reference's own sources (see oracle/Makefile) into
// oracle/_ref/librn_ref.so. Tests and the CPU-baseline leg of bench.py load it
// through ctypes to obtain golden results from the reference itself:
//   * BVH::BVH / BVH::intersect / BVH::occluded      (src/BVH.cpp:6-139)
//   * getClosestIntersection / intersectTriangle     (src/Geometry.cpp:11-63)
//   * renderPathTraced                               (src/Renderer.cpp:1119-1170)
//   * renderRaytraced                                (src/Renderer.cpp:909-948)
//   * renderPhotonMapped                             (src/Renderer.cpp:1300-1349)
//   * renderBidirectional                            (src/BDPT.cpp:65-144)
//   * renderMetropolis                               (src/Metropolis.cpp:85-192)
//   * loadOBJ                                        (src/ObjLoader.cpp:102-214)
// BVH's node array and triangle order are private in the reference; this shim
// exposes them (for dumping the tree it built) by compiling BVH.h with
// `private` mapped to `public`.

#include <cstdint>
#include <cstring>
#include <vector>

#define private public
#include "BVH.h"
#undef private

#include "BDPT.h"
#include "Metropolis.h"

#include "Camera.h"
#include "Geometry.h"
#include "Light.h"
#include "ObjLoader.h"
#include "Renderer.h"
#include <Canvas.h>

namespace {
struct Model {
	std::vector<ModelTriangle> tris;
};
} // namespace

extern "C" {

// ---- triangle lists --------------------------------------------------------

// v9: n*9 floats (v0,v1,v2); rgb: n*3 ints 0..255 (may be null -> white);
// material: n ints in the reference Material enum order (may be null -> Diffuse);
// roughness: n floats (may be null -> 0.2, the reference default);
// normal3: n*3 floats (may be null -> cross(e0, e1) / |cross|, as loadOBJ computes it).
void *refsh_model_new(int n, const float *v9, const int *rgb, const int *material, const float *roughness,
                      const float *normal3) {
	Model *m = new Model();
	m->tris.reserve(static_cast<size_t>(n));
	for (int i = 0; i < n; i++) {
		const float *p = v9 + 9 * static_cast<size_t>(i);
		Colour c = rgb ? Colour(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]) : Colour(255, 255, 255);
		ModelTriangle t(glm::vec3(p[0], p[1], p[2]), glm::vec3(p[3], p[4], p[5]), glm::vec3(p[6], p[7], p[8]), c);
		if (normal3) {
			t.normal = glm::vec3(normal3[3 * i], normal3[3 * i + 1], normal3[3 * i + 2]);
		} else {
			glm::vec3 c = glm::cross(t.vertices[1] - t.vertices[0], t.vertices[2] - t.vertices[0]);
			float len = glm::length(c);
			t.normal = (len > 1e-8f) ? c / len : glm::vec3(0.0f, 1.0f, 0.0f);
		}
		t.vertexNormals = {t.normal, t.normal, t.normal};
		if (material)
			t.material = static_cast<Material>(material[i]);
		if (roughness)
			t.roughness = roughness[i];
		m->tris.push_back(t);
	}
	return m;
}

void *refsh_model_from_obj(const char *path, float scale) {
	Model *m = new Model();
	m->tris = loadOBJ(path, scale);
	return m;
}

int refsh_model_count(const void *h) {
	return static_cast<int>(static_cast<const Model *>(h)->tris.size());
}

// Any output pointer may be null.
void refsh_model_get(const void *h, float *v9, int *rgb, int *material, float *normal3, float *roughness,
                     float *vnormal9) {
	const Model *m = static_cast<const Model *>(h);
	for (size_t i = 0; i < m->tris.size(); i++) {
		const ModelTriangle &t = m->tris[i];
		for (int k = 0; k < 3; k++) {
			if (v9) {
				v9[9 * i + 3 * k + 0] = t.vertices[k].x;
				v9[9 * i + 3 * k + 1] = t.vertices[k].y;
				v9[9 * i + 3 * k + 2] = t.vertices[k].z;
			}
			if (vnormal9) {
				vnormal9[9 * i + 3 * k + 0] = t.vertexNormals[k].x;
				vnormal9[9 * i + 3 * k + 1] = t.vertexNormals[k].y;
				vnormal9[9 * i + 3 * k + 2] = t.vertexNormals[k].z;
			}
		}
		if (rgb) {
			rgb[3 * i] = t.colour.red;
			rgb[3 * i + 1] = t.colour.green;
			rgb[3 * i + 2] = t.colour.blue;
		}
		if (material)
			material[i] = static_cast<int>(t.material);
		if (normal3) {
			normal3[3 * i] = t.normal.x;
			normal3[3 * i + 1] = t.normal.y;
			normal3[3 * i + 2] = t.normal.z;
		}
		if (roughness)
			roughness[i] = t.roughness;
	}
}

// vn9: n*9 floats, the three vertex normals of each triangle (ModelTriangle::vertexNormals).
void refsh_model_set_vertex_normals(void *h, const float *vn9) {
	Model *m = static_cast<Model *>(h);
	for (size_t i = 0; i < m->tris.size(); i++)
		for (int k = 0; k < 3; k++)
			m->tris[i].vertexNormals[k] =
			    glm::vec3(vn9[9 * i + 3 * k], vn9[9 * i + 3 * k + 1], vn9[9 * i + 3 * k + 2]);
}

void refsh_model_free(void *h) {
	delete static_cast<Model *>(h);
}

// ---- BVH ---------------------------------------------------------------------

void *refsh_bvh_new(const void *model) {
	return new BVH(static_cast<const Model *>(model)->tris);
}

void refsh_bvh_free(void *h) {
	delete static_cast<BVH *>(h);
}

int refsh_bvh_node_count(const void *h) {
	return static_cast<int>(static_cast<const BVH *>(h)->nodes.size());
}

int refsh_bvh_root(const void *h) {
	return static_cast<const BVH *>(h)->root;
}

// order: n ints; bounds: nodes*6 floats (bmin, bmax); links: nodes*4 ints (left, right, start, count).
void refsh_bvh_dump(const void *h, int *order, float *bounds, int *links) {
	const BVH *b = static_cast<const BVH *>(h);
	for (size_t i = 0; i < b->order.size(); i++)
		order[i] = b->order[i];
	for (size_t i = 0; i < b->nodes.size(); i++) {
		const auto &nd = b->nodes[i];
		bounds[6 * i + 0] = nd.bmin.x;
		bounds[6 * i + 1] = nd.bmin.y;
		bounds[6 * i + 2] = nd.bmin.z;
		bounds[6 * i + 3] = nd.bmax.x;
		bounds[6 * i + 4] = nd.bmax.y;
		bounds[6 * i + 5] = nd.bmax.z;
		links[4 * i + 0] = nd.left;
		links[4 * i + 1] = nd.right;
		links[4 * i + 2] = nd.start;
		links[4 * i + 3] = nd.count;
	}
}

// Closest hit for n rays. ignore may be null (-1 for all). idx = -1 on a miss.
void refsh_bvh_intersect(const void *h, int n, const float *o3, const float *d3, const int *ignore, int *idx, float *t,
                         float *u, float *v) {
	const BVH *b = static_cast<const BVH *>(h);
#pragma omp parallel for schedule(dynamic, 256)
	for (int i = 0; i < n; i++) {
		glm::vec3 o(o3[3 * i], o3[3 * i + 1], o3[3 * i + 2]);
		glm::vec3 d(d3[3 * i], d3[3 * i + 1], d3[3 * i + 2]);
		RayTriangleIntersection r = b->intersect(o, d, ignore ? ignore[i] : -1);
		idx[i] = r.hit ? static_cast<int>(r.triangleIndex) : -1;
		t[i] = r.distanceFromCamera;
		u[i] = r.u;
		v[i] = r.v;
	}
}

void refsh_bvh_occluded(const void *h, int n, const float *o3, const float *d3, const float *maxd, const int *ignore,
                        int *occ) {
	const BVH *b = static_cast<const BVH *>(h);
#pragma omp parallel for schedule(dynamic, 256)
	for (int i = 0; i < n; i++) {
		glm::vec3 o(o3[3 * i], o3[3 * i + 1], o3[3 * i + 2]);
		glm::vec3 d(d3[3 * i], d3[3 * i + 1], d3[3 * i + 2]);
		occ[i] = b->occluded(o, d, maxd[i], ignore ? ignore[i] : -1) ? 1 : 0;
	}
}

// Brute-force closest hit (getClosestIntersection) for n rays.
void refsh_brute_intersect(const void *model, int n, const float *o3, const float *d3, int *idx, float *t) {
	const Model *m = static_cast<const Model *>(model);
#pragma omp parallel for schedule(dynamic, 64)
	for (int i = 0; i < n; i++) {
		glm::vec3 o(o3[3 * i], o3[3 * i + 1], o3[3 * i + 2]);
		glm::vec3 d(d3[3 * i], d3[3 * i + 1], d3[3 * i + 2]);
		RayTriangleIntersection r = getClosestIntersection(o, d, m->tris);
		idx[i] = r.hit ? static_cast<int>(r.triangleIndex) : -1;
		t[i] = r.distanceFromCamera;
	}
}

// One ray against one triangle: returns 1 on a hit and writes t, u, v.
int refsh_intersect_triangle(const float *o3, const float *d3, const float *v9, float *t, float *u, float *v) {
	ModelTriangle tri(glm::vec3(v9[0], v9[1], v9[2]), glm::vec3(v9[3], v9[4], v9[5]), glm::vec3(v9[6], v9[7], v9[8]),
	                  Colour());
	return intersectTriangle(glm::vec3(o3[0], o3[1], o3[2]), glm::vec3(d3[0], d3[1], d3[2]), tri, *t, *u, *v) ? 1 : 0;
}

// ---- renderPathTraced ---------------------------------------------------------

// Light records: 24 floats each --
// [type, pos3, dir3, colour3, intensity, radius, coneCos, kc, kl, kq, u3, v3, pad2]
static std::vector<Light> unpackLights(int n, const float *rec) {
	std::vector<Light> out;
	for (int i = 0; i < n; i++) {
		const float *r = rec + 24 * static_cast<size_t>(i);
		Light L;
		L.type = static_cast<LightType>(static_cast<int>(r[0]));
		L.position = glm::vec3(r[1], r[2], r[3]);
		L.direction = glm::vec3(r[4], r[5], r[6]);
		L.colour = glm::vec3(r[7], r[8], r[9]);
		L.intensity = r[10];
		L.radius = r[11];
		L.coneCos = r[12];
		L.attenConstant = r[13];
		L.attenLinear = r[14];
		L.attenQuadratic = r[15];
		L.uAxis = glm::vec3(r[16], r[17], r[18]);
		L.vAxis = glm::vec3(r[19], r[20], r[21]);
		out.push_back(L);
	}
	return out;
}

// Camera(w, h, focal, pos) + lookAt(target), exactly as the C ABI builds it
// (src/capi.cpp:49-50) but with the position/target/focal exposed.
// Output: w*h uint32 0xAARRGGBB, the reference Canvas format.
void refsh_render_pathtraced(const void *model, int w, int h, float focal, const float *pos3, const float *target3,
                             int samples, int n_lights, const float *lights, float aperture, float focus,
                             const float *motion3, int blades, uint32_t *out) {
	const Model *m = static_cast<const Model *>(model);
	Camera cam(w, h, focal, glm::vec3(pos3[0], pos3[1], pos3[2]));
	cam.lookAt(glm::vec3(target3[0], target3[1], target3[2]));
	Canvas canvas(static_cast<size_t>(w), static_cast<size_t>(h));
	glm::vec3 motion = motion3 ? glm::vec3(motion3[0], motion3[1], motion3[2]) : glm::vec3(0.0f);
	renderPathTraced(m->tris, cam, canvas, samples, unpackLights(n_lights, lights), aperture, focus, motion, {},
	                 blades);
	std::memcpy(out, canvas.pixels.data(), sizeof(uint32_t) * static_cast<size_t>(w) * static_cast<size_t>(h));
}

// renderRaytraced with the camera built as renderPathTraced's above; shading is the
// ShadingModel value (0 flat, 1 Gouraud, 2 Phong); fog3 may be null (the default colour).
void refsh_render_raytraced(const void *model, int w, int h, float focal, const float *pos3, const float *target3,
                            int shading, int n_lights, const float *lights, float fog_density, const float *fog3,
                            uint32_t *out) {
	const Model *m = static_cast<const Model *>(model);
	Camera cam(w, h, focal, glm::vec3(pos3[0], pos3[1], pos3[2]));
	cam.lookAt(glm::vec3(target3[0], target3[1], target3[2]));
	Canvas canvas(static_cast<size_t>(w), static_cast<size_t>(h));
	const glm::vec3 fog = fog3 ? glm::vec3(fog3[0], fog3[1], fog3[2]) : glm::vec3(200.0f, 210.0f, 230.0f);
	renderRaytraced(m->tris, cam, canvas, static_cast<ShadingModel>(shading), unpackLights(n_lights, lights), {},
	                fog_density, fog);
	std::memcpy(out, canvas.pixels.data(), sizeof(uint32_t) * static_cast<size_t>(w) * static_cast<size_t>(h));
}

// renderPhotonMapped with the camera built as above (src/Renderer.cpp:1300-1349).
void refsh_render_photon_mapped(const void *model, int w, int h, float focal, const float *pos3, const float *target3,
                                int num_photons, int gather_rays, int n_lights, const float *lights, uint32_t *out) {
	const Model *m = static_cast<const Model *>(model);
	Camera cam(w, h, focal, glm::vec3(pos3[0], pos3[1], pos3[2]));
	cam.lookAt(glm::vec3(target3[0], target3[1], target3[2]));
	Canvas canvas(static_cast<size_t>(w), static_cast<size_t>(h));
	renderPhotonMapped(m->tris, cam, canvas, num_photons, unpackLights(n_lights, lights), {}, gather_rays);
	std::memcpy(out, canvas.pixels.data(), sizeof(uint32_t) * static_cast<size_t>(w) * static_cast<size_t>(h));
}

// renderBidirectional / renderMetropolis with the camera built as above.
void refsh_render_bidirectional(const void *model, int w, int h, float focal, const float *pos3, const float *target3,
                                int samples, float exposure, uint32_t *out) {
	const Model *m = static_cast<const Model *>(model);
	Camera cam(w, h, focal, glm::vec3(pos3[0], pos3[1], pos3[2]));
	cam.lookAt(glm::vec3(target3[0], target3[1], target3[2]));
	Canvas canvas(static_cast<size_t>(w), static_cast<size_t>(h));
	renderBidirectional(m->tris, cam, canvas, samples, exposure);
	std::memcpy(out, canvas.pixels.data(), sizeof(uint32_t) * static_cast<size_t>(w) * static_cast<size_t>(h));
}

void refsh_render_metropolis(const void *model, int w, int h, float focal, const float *pos3, const float *target3,
                             int mutations, float exposure, uint32_t *out) {
	const Model *m = static_cast<const Model *>(model);
	Camera cam(w, h, focal, glm::vec3(pos3[0], pos3[1], pos3[2]));
	cam.lookAt(glm::vec3(target3[0], target3[1], target3[2]));
	Canvas canvas(static_cast<size_t>(w), static_cast<size_t>(h));
	renderMetropolis(m->tris, cam, canvas, mutations, exposure);
	std::memcpy(out, canvas.pixels.data(), sizeof(uint32_t) * static_cast<size_t>(w) * static_cast<size_t>(h));
}

// ---- canvas post-processing (src/Renderer.cpp:1353-1470), in place on px ----
static Canvas to_canvas(const uint32_t *px, int w, int h) {
	Canvas c(static_cast<size_t>(w), static_cast<size_t>(h));
	std::memcpy(c.pixels.data(), px, sizeof(uint32_t) * static_cast<size_t>(w) * static_cast<size_t>(h));
	return c;
}
static void from_canvas(const Canvas &c, uint32_t *px) {
	std::memcpy(px, c.pixels.data(), sizeof(uint32_t) * c.pixels.size());
}
void refsh_tonemap(uint32_t *px, int w, int h, float exposure, float gamma) {
	Canvas c = to_canvas(px, w, h);
	toneMap(c, exposure, gamma);
	from_canvas(c, px);
}
void refsh_bloom(uint32_t *px, int w, int h, float threshold, float intensity) {
	Canvas c = to_canvas(px, w, h);
	applyBloom(c, threshold, intensity);
	from_canvas(c, px);
}
void refsh_fxaa(uint32_t *px, int w, int h) {
	Canvas c = to_canvas(px, w, h);
	applyFXAA(c);
	from_canvas(c, px);
}
// AccumBuffer over n_frames canvases stored one after another; the resolve into out.
void refsh_accum(int n_frames, const uint32_t *frames, int w, int h, uint32_t *out) {
	AccumBuffer acc(w, h);
	const size_t n = static_cast<size_t>(w) * static_cast<size_t>(h);
	for (int f = 0; f < n_frames; f++)
		acc.add(to_canvas(frames + n * static_cast<size_t>(f), w, h));
	Canvas c(static_cast<size_t>(w), static_cast<size_t>(h));
	acc.resolve(c);
	from_canvas(c, out);
}

} // extern "C"
