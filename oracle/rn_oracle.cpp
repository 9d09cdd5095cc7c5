// TEST INFRASTRUCTURE ONLY -- the CPU oracle. Never linked into the product.
//
// An independent CPU restatement of the reference path tracer's hot path, used
// by tests/ (and the CPU-baseline leg of bench.py) to check the CUDA kernels.
// It is pinned against the reference itself (oracle/_ref/librn_ref.so, built
// from the reference sources) by the CPU tests in tests/test_oracle.py.
//
// Restated here, each from the cited reference lines:
//   * BVH build, median split, leaf <= 4           src/BVH.cpp:6-63
//   * slab test                                     src/BVH.cpp:66-75
//   * closest hit / any hit traversal               src/BVH.cpp:77-139
//   * ray/triangle test (glm inverse order)         src/Geometry.cpp:11-25
//   * reference path-tracer estimator               src/Renderer.cpp:390-498, 555-563,
//                                                   642-660, 775-907, 1103-1170
//   * improved Perlin noise (procedural colour)     src/Noise.cpp:6-61, 246-255
// The traversal is instrumented: it counts node box tests and triangle tests,
// which give the algorithmic bytes of a ray query (24 B per box, 36 B per
// triangle) used as the roofline numerator.
//
// Built with -ffp-contract=off (oracle/Makefile): no FMA contraction, so float
// results follow the reference's non-FMA build operation by operation.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#include "rn_oracle_rng.hpp"

namespace {

struct V3 {
	float x, y, z;
};
inline V3 mk(float x, float y, float z) { return {x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float dot(V3 a, V3 b) {
	float x = a.x * b.x, y = a.y * b.y, z = a.z * b.z;
	return (x + y) + z;
}
inline V3 cross(V3 x, V3 y) { return {x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y}; }
inline float length(V3 v) { return std::sqrt(dot(v, v)); }
inline V3 normalize(V3 v) { return v * (1.0f / std::sqrt(dot(v, v))); }
inline V3 reflect(V3 I, V3 N) { return I - (N * dot(N, I)) * 2.0f; }
inline V3 refract(V3 I, V3 N, float eta) {
	float dv = dot(N, I);
	float k = 1.0f - eta * eta * (1.0f - dv * dv);
	return (k >= 0.0f) ? (eta * I - (eta * dv + std::sqrt(k)) * N) : mk(0, 0, 0);
}
inline V3 mix(V3 x, V3 y, float a) { return x * (1.0f - a) + y * a; }
inline float gmin(float x, float y) { return (y < x) ? y : x; }
inline float gmax(float x, float y) { return (x < y) ? y : x; }
inline V3 vmin(V3 a, V3 b) { return {gmin(a.x, b.x), gmin(a.y, b.y), gmin(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return {gmax(a.x, b.x), gmax(a.y, b.y), gmax(a.z, b.z)}; }
inline float comp(V3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

struct Tri {
	V3 v0, v1, v2;
};

struct Node {
	V3 bmin, bmax;
	int left = -1, right = -1, start = 0, count = 0;
};

struct Bvh {
	std::vector<Tri> tris;
	std::vector<V3> cent;
	std::vector<int> order;
	std::vector<Node> nodes;
	int root = -1;

	int build(int start, int count) {
		Node node;
		V3 lo = mk(1e30f, 1e30f, 1e30f), hi = mk(-1e30f, -1e30f, -1e30f);
		for (int i = start; i < start + count; i++) {
			const Tri &t = tris[order[i]];
			for (V3 v : {t.v0, t.v1, t.v2}) {
				lo = vmin(lo, v);
				hi = vmax(hi, v);
			}
		}
		node.bmin = lo;
		node.bmax = hi;
		if (count <= 4) {
			node.start = start;
			node.count = count;
			nodes.push_back(node);
			return static_cast<int>(nodes.size()) - 1;
		}
		V3 cmin = mk(1e30f, 1e30f, 1e30f), cmax = mk(-1e30f, -1e30f, -1e30f);
		for (int i = start; i < start + count; i++) {
			cmin = vmin(cmin, cent[order[i]]);
			cmax = vmax(cmax, cent[order[i]]);
		}
		V3 e = cmax - cmin;
		int axis = (e.x > e.y && e.x > e.z) ? 0 : (e.y > e.z ? 1 : 2);
		int mid = start + count / 2;
		std::nth_element(order.begin() + start, order.begin() + mid, order.begin() + start + count,
		                 [&](int a, int b) { return comp(cent[a], axis) < comp(cent[b], axis); });
		if (mid == start || mid == start + count) {
			node.start = start;
			node.count = count;
			nodes.push_back(node);
			return static_cast<int>(nodes.size()) - 1;
		}
		int self = static_cast<int>(nodes.size());
		nodes.push_back(node);
		int l = build(start, mid - start);
		int r = build(mid, start + count - mid);
		nodes[self].left = l;
		nodes[self].right = r;
		return self;
	}
};

bool slab_hit(V3 o, V3 inv, V3 lo, V3 hi, float tmax) {
	V3 t0 = (lo - o) * inv, t1 = (hi - o) * inv;
	V3 ts = vmin(t0, t1), tb = vmax(t0, t1);
	float te = ts.x;
	if (te < ts.y)
		te = ts.y;
	if (te < ts.z)
		te = ts.z;
	float tx = tb.x;
	if (tb.y < tx)
		tx = tb.y;
	if (tb.z < tx)
		tx = tb.z;
	float m0 = (te < 0.0f) ? 0.0f : te;
	return tx >= m0 && te < tmax;
}

// inverse(mat3(-d, e0, e1)) * (o - v0) in glm's expression order.
bool tri_hit(V3 o, V3 d, const Tri &tr, float &t, float &u, float &v) {
	V3 e0 = tr.v1 - tr.v0, e1 = tr.v2 - tr.v0, sp = o - tr.v0;
	V3 m0 = -d, m1 = e0, m2 = e1;
	float det = +m0.x * (m1.y * m2.z - m2.y * m1.z) - m1.x * (m0.y * m2.z - m2.y * m0.z) +
	            m2.x * (m0.y * m1.z - m1.y * m0.z);
	if (std::fabs(det) < 1e-8f)
		return false;
	float k = 1.0f / (+m0.x * (m1.y * m2.z - m2.y * m1.z) - m1.x * (m0.y * m2.z - m2.y * m0.z) +
	                  m2.x * (m0.y * m1.z - m1.y * m0.z));
	float i00 = +(m1.y * m2.z - m2.y * m1.z) * k;
	float i10 = -(m1.x * m2.z - m2.x * m1.z) * k;
	float i20 = +(m1.x * m2.y - m2.x * m1.y) * k;
	float i01 = -(m0.y * m2.z - m2.y * m0.z) * k;
	float i11 = +(m0.x * m2.z - m2.x * m0.z) * k;
	float i21 = -(m0.x * m2.y - m2.x * m0.y) * k;
	float i02 = +(m0.y * m1.z - m1.y * m0.z) * k;
	float i12 = -(m0.x * m1.z - m1.x * m0.z) * k;
	float i22 = +(m0.x * m1.y - m1.x * m0.y) * k;
	t = i00 * sp.x + i10 * sp.y + i20 * sp.z;
	u = i01 * sp.x + i11 * sp.y + i21 * sp.z;
	v = i02 * sp.x + i12 * sp.y + i22 * sp.z;
	return (u >= 0.0f) && (v >= 0.0f) && (u + v <= 1.0f) && (t > 1e-5f);
}

struct Counts {
	long boxes = 0, tris = 0;
};

struct Hit {
	bool hit = false;
	int idx = -1;
	float t = INFINITY, u = 0, v = 0;
	V3 point = mk(0, 0, 0);
};

Hit intersect(const Bvh &b, V3 o, V3 d, int ignore, Counts *cnt) {
	Hit h;
	if (b.root < 0)
		return h;
	V3 inv = mk(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
	int st[64], sp = 0;
	st[sp++] = b.root;
	while (sp > 0) {
		const Node &n = b.nodes[st[--sp]];
		if (cnt)
			cnt->boxes++;
		if (!slab_hit(o, inv, n.bmin, n.bmax, h.t))
			continue;
		if (n.count > 0) {
			for (int i = n.start; i < n.start + n.count; i++) {
				int ti = b.order[i];
				if (ti == ignore)
					continue;
				float t, u, v;
				if (cnt)
					cnt->tris++;
				if (tri_hit(o, d, b.tris[ti], t, u, v) && t < h.t) {
					h.hit = true;
					h.idx = ti;
					h.t = t;
					h.u = u;
					h.v = v;
					h.point = o + t * d;
				}
			}
		} else {
			st[sp++] = n.left;
			st[sp++] = n.right;
		}
	}
	return h;
}

bool occluded(const Bvh &b, V3 o, V3 d, float maxd, int ignore, Counts *cnt) {
	if (b.root < 0)
		return false;
	V3 inv = mk(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
	int st[64], sp = 0;
	st[sp++] = b.root;
	while (sp > 0) {
		const Node &n = b.nodes[st[--sp]];
		if (cnt)
			cnt->boxes++;
		if (!slab_hit(o, inv, n.bmin, n.bmax, maxd))
			continue;
		if (n.count > 0) {
			for (int i = n.start; i < n.start + n.count; i++) {
				int ti = b.order[i];
				if (ti == ignore)
					continue;
				float t, u, v;
				if (cnt)
					cnt->tris++;
				if (tri_hit(o, d, b.tris[ti], t, u, v) && t < maxd)
					return true;
			}
		} else {
			st[sp++] = n.left;
			st[sp++] = n.right;
		}
	}
	return false;
}

// ---- reference-mode estimator ------------------------------------------------

struct RefTri {
	V3 normal;
	int material;
	V3 rgb;
	float roughness;
};

struct Light {
	int type;
	V3 pos, dir, colour;
	float intensity, radius, cone_cos, kc, kl, kq;
	V3 u, v;
};

enum { kDiffuse = 0, kMirror, kGlass, kProcedural, kBump, kParallax, kMetal, kDispersive, kSubsurface, kNormalMap,
       kEmissive };
enum { kPoint = 0, kDirectional, kSpot, kVolume, kRectangle, kTriangle };

const int kPerm[256] = {
    151, 160, 137, 91,  90,  15,  131, 13,  201, 95,  96,  53,  194, 233, 7,   225, 140, 36,  103, 30,  69,  142,
    8,   99,  37,  240, 21,  10,  23,  190, 6,   148, 247, 120, 234, 75,  0,   26,  197, 62,  94,  252, 219, 203,
    117, 35,  11,  32,  57,  177, 33,  88,  237, 149, 56,  87,  174, 20,  125, 136, 171, 168, 68,  175, 74,  165,
    71,  134, 139, 48,  27,  166, 77,  146, 158, 231, 83,  111, 229, 122, 60,  211, 133, 230, 220, 105, 92,  41,
    55,  46,  245, 40,  244, 102, 143, 54,  65,  25,  63,  161, 1,   216, 80,  73,  209, 76,  132, 187, 208, 89,
    18,  169, 200, 196, 135, 130, 116, 188, 159, 86,  164, 100, 109, 198, 173, 186, 3,   64,  52,  217, 226, 250,
    124, 123, 5,   202, 38,  147, 118, 126, 255, 82,  85,  212, 207, 206, 59,  227, 47,  16,  58,  17,  182, 189,
    28,  42,  223, 183, 170, 213, 119, 248, 152, 2,   44,  154, 163, 70,  221, 153, 101, 155, 167, 43,  172, 9,
    129, 22,  39,  253, 19,  98,  108, 110, 79,  113, 224, 232, 178, 185, 112, 104, 218, 246, 97,  228, 251, 34,
    242, 193, 238, 210, 144, 12,  191, 179, 162, 241, 81,  51,  145, 235, 249, 14,  239, 107, 49,  192, 214, 31,
    181, 199, 106, 157, 184, 84,  204, 176, 115, 121, 50,  45,  127, 4,   150, 254, 138, 236, 205, 93,  222, 114,
    67,  29,  24,  72,  243, 141, 128, 195, 78,  66,  215, 61,  156, 180};
inline int P(int i) { return kPerm[i & 255]; }
inline float fade(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }
inline float plerp(float t, float a, float b) { return a + t * (b - a); }
inline float grad(int hash, float x, float y, float z) {
	int h = hash & 15;
	float u = h < 8 ? x : y;
	float v = h < 4 ? y : (h == 12 || h == 14 ? x : z);
	return ((h & 1) == 0 ? u : -u) + ((h & 2) == 0 ? v : -v);
}
float perlin(float x, float y, float z) {
	int X = static_cast<int>(std::floor(x)) & 255, Y = static_cast<int>(std::floor(y)) & 255,
	    Z = static_cast<int>(std::floor(z)) & 255;
	x -= std::floor(x);
	y -= std::floor(y);
	z -= std::floor(z);
	float u = fade(x), v = fade(y), w = fade(z);
	int A = P(X) + Y, AA = P(A) + Z, AB = P(A + 1) + Z;
	int B = P(X + 1) + Y, BA = P(B) + Z, BB = P(B + 1) + Z;
	return plerp(w,
	             plerp(v, plerp(u, grad(P(AA), x, y, z), grad(P(BA), x - 1, y, z)),
	                   plerp(u, grad(P(AB), x, y - 1, z), grad(P(BB), x - 1, y - 1, z))),
	             plerp(v, plerp(u, grad(P(AA + 1), x, y, z - 1), grad(P(BA + 1), x - 1, y, z - 1)),
	                   plerp(u, grad(P(AB + 1), x, y - 1, z - 1), grad(P(BB + 1), x - 1, y - 1, z - 1))));
}
V3 procedural(V3 p) {
	V3 q = p * 3.0f;
	float sum = 0.0f, amp = 1.0f, freq = 1.0f, norm = 0.0f;
	for (int i = 0; i < 4; i++) {
		sum += amp * perlin(q.x * freq, q.y * freq, q.z * freq);
		norm += amp;
		amp *= 0.5f;
		freq *= 2.0f;
	}
	float n = 0.5f + 0.5f * (sum / norm);
	float rings = 0.5f + 0.5f * std::sin((q.x + q.y) * 3.0f + n * 8.0f);
	return mix(mk(60, 30, 12), mk(205, 150, 90), rings);
}

struct RefScene {
	const Bvh *bvh;
	std::vector<RefTri> tri;
	std::vector<Light> lights;
	int max_depth;
};

float visibility(const RefScene &s, const Light &L, V3 p, int ig) {
	const Bvh &b = *s.bvh;
	if (L.type == kDirectional)
		return occluded(b, p, -normalize(L.dir), 1e6f, ig, nullptr) ? 0.0f : 1.0f;
	auto frac = [&](V3 sp) {
		V3 to = sp - p;
		float dist = length(to);
		return occluded(b, p, to / dist, dist, ig, nullptr) ? 0 : 1;
	};
	if (L.type == kRectangle) {
		const float g[9][2] = {{-1, -1}, {0, -1}, {1, -1}, {-1, 0}, {0, 0}, {1, 0}, {-1, 1}, {0, 1}, {1, 1}};
		int u = 0;
		for (auto &q : g)
			u += frac(L.pos + L.u * q[0] + L.v * q[1]);
		return u / 9.0f;
	}
	if (L.type == kTriangle) {
		const float g[9][2] = {{0, 0}, {1, 0}, {0, 1}, {0.5f, 0}, {0, 0.5f}, {0.5f, 0.5f}, {0.25f, 0.25f},
		                       {0.5f, 0.25f}, {1.0f / 3.0f, 1.0f / 3.0f}};
		int u = 0;
		for (auto &q : g)
			u += frac(L.pos + L.u * q[0] + L.v * q[1]);
		return u / 9.0f;
	}
	if (L.radius <= 0.0f)
		return static_cast<float>(frac(L.pos));
	if (L.type == kVolume) {
		const float kPi = 3.14159265358979323846f;
		V3 toc = L.pos - p;
		float d = length(toc);
		V3 dir = toc / d;
		float smx = std::min(1.0f, L.radius / d);
		if (smx >= 1.0f)
			return 1.0f;
		float cmx = std::sqrt(std::max(0.0f, 1.0f - smx * smx));
		V3 up = std::fabs(dir.y) < 0.99f ? mk(0, 1, 0) : mk(1, 0, 0);
		V3 tg = normalize(cross(up, dir)), bt = cross(dir, tg);
		const float rc[2] = {0.85f, 0.4f}, ro[2] = {0.0f, 0.5f};
		const int rn[2] = {5, 6};
		int un = 0, tot = 1;
		if (!occluded(b, p, dir, d, ig, nullptr))
			un++;
		for (int r = 0; r < 2; r++) {
			float ct = 1.0f - rc[r] * (1.0f - cmx), st = std::sqrt(std::max(0.0f, 1.0f - ct * ct));
			for (int i = 0; i < rn[r]; i++) {
				float phi = 2.0f * kPi * ((static_cast<float>(i) + ro[r]) / static_cast<float>(rn[r]));
				V3 sd = normalize(dir * ct + (tg * std::cos(phi) + bt * std::sin(phi)) * st);
				if (!occluded(b, p, sd, d, ig, nullptr))
					un++;
				tot++;
			}
		}
		return static_cast<float>(un) / static_cast<float>(tot);
	}
	const float ks[9][2] = {{0, 0}, {1, 0}, {-1, 0}, {0, 1}, {0, -1}, {0.7f, 0.7f}, {-0.7f, 0.7f}, {0.7f, -0.7f},
	                        {-0.7f, -0.7f}};
	V3 axis = normalize(p - L.pos);
	V3 up = std::fabs(axis.y) < 0.99f ? mk(0, 1, 0) : mk(1, 0, 0);
	V3 tg = normalize(cross(up, axis)), bt = cross(axis, tg);
	int u = 0;
	for (auto &q : ks)
		u += frac(L.pos + (tg * q[0] + bt * q[1]) * L.radius);
	return u / 9.0f;
}

void light_dir(const Light &L, V3 p, V3 &dir, float &att) {
	if (L.type == kDirectional) {
		dir = -normalize(L.dir);
		att = L.intensity / 40.0f;
	} else {
		V3 to = L.pos - p;
		float dist = length(to);
		dir = to / dist;
		att = L.intensity / (L.kc + L.kl * dist + L.kq * dist * dist);
	}
}

V3 direct_light(const RefScene &s, V3 p, V3 n, V3 albedo, int ig) {
	V3 sum = mk(0, 0, 0);
	for (const Light &L : s.lights) {
		V3 ld;
		float att;
		light_dir(L, p, ld, att);
		float cone = 1.0f;
		if (L.type == kSpot)
			cone = (dot(-ld, normalize(L.dir)) > L.cone_cos) ? 1.0f : 0.0f;
		float vis = visibility(s, L, p, ig);
		float inc = std::max(0.0f, dot(n, ld));
		sum = sum + L.colour * (vis * cone * att * inc);
	}
	return albedo * vmin(sum, mk(1, 1, 1));
}

using Rng = std::mt19937;
float U01(Rng &r) { return std::uniform_real_distribution<float>(0.0f, 1.0f)(r); }

V3 cosine_hemisphere(V3 n, Rng &rng) {
	float u1 = U01(rng), u2 = U01(rng);
	float r = std::sqrt(u1), th = 2.0f * 3.14159265f * u2;
	float x = r * std::cos(th), y = r * std::sin(th), z = std::sqrt(std::max(0.0f, 1.0f - u1));
	V3 up = std::fabs(n.z) < 0.99f ? mk(0, 0, 1) : mk(1, 0, 0);
	V3 t = normalize(cross(up, n)), b = cross(n, t);
	return normalize(t * x + b * y + n * z);
}

V3 face_viewer(V3 n, V3 d) { return dot(n, d) > 0.0f ? -n : n; }

V3 base_colour(const RefTri &t, V3 p) { return t.material == kProcedural ? procedural(p) : t.rgb; }

V3 path_trace(const RefScene &s, V3 o, V3 d, int depth, Rng &rng) {
	Hit h = intersect(*s.bvh, o, d, -1, nullptr);
	if (!h.hit) {
		float t = 0.5f * (d.y + 1.0f);
		return mix(mk(200, 210, 235), mk(70, 120, 205), t) / 255.0f;
	}
	const RefTri &tr = s.tri[h.idx];
	V3 p = h.point;
	int ig = h.idx;
	if (tr.material == kEmissive)
		return tr.rgb / 255.0f * 4.0f;
	if (tr.material == kMirror && depth > 0) {
		V3 n = face_viewer(tr.normal, d), r = reflect(d, n);
		return path_trace(s, p + 1e-4f * r, r, depth - 1, rng);
	}
	if ((tr.material == kGlass || tr.material == kDispersive) && depth > 0) {
		V3 n = tr.normal;
		float cosi = dot(d, n), etai = 1.0f, etat = 1.5f;
		if (cosi < 0.0f) {
			cosi = -cosi;
		} else {
			std::swap(etai, etat);
			n = -n;
		}
		float r0 = (etai - etat) / (etai + etat);
		r0 *= r0;
		float fr = r0 + (1.0f - r0) * std::pow(1.0f - cosi, 5.0f);
		V3 rf = refract(d, n, etai / etat);
		V3 dir = (length(rf) < 1e-6f || U01(rng) < fr) ? reflect(d, n) : rf;
		return path_trace(s, p + 1e-4f * dir, dir, depth - 1, rng);
	}
	if (tr.material == kMetal && depth > 0) {
		V3 n = face_viewer(tr.normal, d), r = reflect(d, n);
		V3 df = cosine_hemisphere(n, rng);
		float r2 = tr.roughness * tr.roughness;
		V3 dir = normalize(mix(r, df, r2));
		if (dot(dir, n) <= 0.0f)
			dir = r;
		V3 albedo = base_colour(tr, p) / 255.0f;
		return albedo * path_trace(s, p + 1e-4f * dir, dir, depth - 1, rng);
	}
	if (tr.material == kSubsurface) {
		V3 n = face_viewer(tr.normal, d);
		V3 albedo = base_colour(tr, p) / 255.0f;
		V3 shade = mk(0, 0, 0);
		for (const Light &L : s.lights) {
			V3 to = L.pos - p;
			float dist = length(to);
			V3 ld = to / dist;
			float att = L.intensity / (L.kc + L.kl * dist + L.kq * dist * dist);
			float wd = std::max(0.0f, (dot(n, ld) + 0.5f) / (1.0f + 0.5f));
			shade = shade + albedo * L.colour * (visibility(s, L, p, ig) * att * wd);
			Hit ex = intersect(*s.bvh, p - n * 1e-3f, ld, ig, nullptr);
			float th = ex.hit ? ex.t : 0.0f;
			shade = shade + albedo * L.colour * (att * std::exp(-3.0f * th) * 0.6f);
		}
		V3 direct = vmin(shade, mk(1.5f, 1.5f, 1.5f));
		if (depth <= 0)
			return direct;
		V3 sb = cosine_hemisphere(n, rng);
		return direct + albedo * path_trace(s, p + 1e-4f * sb, sb, depth - 1, rng);
	}
	V3 n = face_viewer(tr.normal, d);
	V3 albedo = base_colour(tr, p) / 255.0f;
	V3 direct = direct_light(s, p, n, albedo, ig);
	if (depth <= 0)
		return direct;
	V3 bnc = cosine_hemisphere(n, rng);
	return direct + albedo * path_trace(s, p + 1e-4f * bnc, bnc, depth - 1, rng);
}


// ---- physical-mode estimator (templated on the float type) ----------------------
// Restates rednoise_b200's physical estimator (rednoise_b200/csrc/physical.cuh):
// same camera, counter-based uniforms, BSDFs, MIS and roulette. With T = float the
// closest hits come from the reference-exact traversal above; with T = double the
// same BVH is traversed with a double-precision Moller-Trumbore test.

template <typename T> struct X3 {
	T x, y, z;
};
template <typename T> inline X3<T> x3(T a, T b, T c) { return {a, b, c}; }
template <typename T> inline X3<T> operator+(X3<T> a, X3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T> inline X3<T> operator-(X3<T> a, X3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T> inline X3<T> operator-(X3<T> a) { return {-a.x, -a.y, -a.z}; }
template <typename T> inline X3<T> operator*(X3<T> a, X3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <typename T> inline X3<T> operator*(X3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <typename T> inline T dt(X3<T> a, X3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> inline X3<T> cr(X3<T> a, X3<T> b) {
	return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename T> inline X3<T> nz(X3<T> a) { return a * (T(1) / std::sqrt(dt(a, a))); }
template <typename T> inline T mx(X3<T> a) { return std::max(a.x, std::max(a.y, a.z)); }

struct PhysScene {
	Bvh bvh;
	std::vector<float> albedo, emission, param, normal; // 3, 3, 1, 3 per triangle
	std::vector<int> material;
	struct Em {
		float v0[3], e0[3], e1[3];
		float area, cdf;
		int tri;
	};
	std::vector<Em> em;
	float area_total = 0.0f;
};

struct PhysCam {
	float pos[3], fwd[3], right[3], up[3];
	float tan_half, aspect;
	int w, h;
};

struct PhysSet {
	int spp, max_depth, rr_depth;
	uint64_t seed;
	uint32_t offset;
	float env[3];
};

inline orc::U4 prand(uint64_t seed, uint32_t pix, uint32_t s, uint32_t block) {
	return orc::philox4x32_10(orc::U4{pix, s, block, 0u}, static_cast<uint32_t>(seed),
	                          static_cast<uint32_t>(seed >> 32));
}

template <typename T> struct PHit {
	int idx = -1;
	T t = T(0);
};

// Double-precision closest hit over the same tree (nearest-first not needed: full DFS).
PHit<double> closest_d(const PhysScene &s, X3<double> o, X3<double> d, int ignore) {
	PHit<double> h;
	h.t = INFINITY;
	const Bvh &b = s.bvh;
	if (b.root < 0)
		return h;
	X3<double> inv = x3(1.0 / d.x, 1.0 / d.y, 1.0 / d.z);
	int st[64], sp = 0;
	st[sp++] = b.root;
	while (sp > 0) {
		const Node &n = b.nodes[st[--sp]];
		double t0x = (n.bmin.x - o.x) * inv.x, t1x = (n.bmax.x - o.x) * inv.x;
		double t0y = (n.bmin.y - o.y) * inv.y, t1y = (n.bmax.y - o.y) * inv.y;
		double t0z = (n.bmin.z - o.z) * inv.z, t1z = (n.bmax.z - o.z) * inv.z;
		double te = std::max(std::max(std::min(t0x, t1x), std::min(t0y, t1y)), std::min(t0z, t1z));
		double tx = std::min(std::min(std::max(t0x, t1x), std::max(t0y, t1y)), std::max(t0z, t1z));
		if (std::isnan(te) || std::isnan(tx))
			te = 0, tx = INFINITY; // degenerate slab: visit conservatively
		if (!(tx >= std::max(te, 0.0) * (1 - 1e-9) && te <= h.t))
			continue;
		if (n.count > 0) {
			for (int i = n.start; i < n.start + n.count; i++) {
				int ti = b.order[i];
				if (ti == ignore)
					continue;
				const Tri &tr = b.tris[ti];
				X3<double> v0 = x3<double>(tr.v0.x, tr.v0.y, tr.v0.z);
				X3<double> e1 = x3<double>(tr.v1.x, tr.v1.y, tr.v1.z) - v0;
				X3<double> e2 = x3<double>(tr.v2.x, tr.v2.y, tr.v2.z) - v0;
				X3<double> p = cr(d, e2);
				double det = dt(e1, p);
				if (std::fabs(det) < 1e-18)
					continue;
				double id = 1.0 / det;
				X3<double> tv = o - v0;
				double u = dt(tv, p) * id;
				if (u < 0 || u > 1)
					continue;
				X3<double> q = cr(tv, e1);
				double v = dt(d, q) * id;
				if (v < 0 || u + v > 1)
					continue;
				double t = dt(e2, q) * id;
				if (t > 1e-5 && t < h.t) {
					h.t = t;
					h.idx = ti;
				}
			}
		} else {
			st[sp++] = n.left;
			st[sp++] = n.right;
		}
	}
	return h;
}

bool occluded_d(const PhysScene &s, X3<double> o, X3<double> d, double tmax, int ignore) {
	PHit<double> h = closest_d(s, o, d, ignore);
	return h.idx >= 0 && h.t < tmax;
}

// Optional per-thread counters of the reference-order queries (algorithmic bytes).
struct QueryCounts {
	long closest = 0, any = 0;
	Counts cb, ab;
};
thread_local QueryCounts *g_qc = nullptr;

template <typename T> PHit<T> closest_t(const PhysScene &s, X3<T> o, X3<T> d, int ignore);
template <> PHit<float> closest_t<float>(const PhysScene &s, X3<float> o, X3<float> d, int ignore) {
	if (g_qc)
		g_qc->closest++;
	Hit h = intersect(s.bvh, mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), ignore, g_qc ? &g_qc->cb : nullptr);
	PHit<float> r;
	r.idx = h.hit ? h.idx : -1;
	r.t = h.t;
	return r;
}
template <> PHit<double> closest_t<double>(const PhysScene &s, X3<double> o, X3<double> d, int ignore) {
	return closest_d(s, o, d, ignore);
}
template <typename T> bool occluded_t(const PhysScene &s, X3<T> o, X3<T> d, T tmax, int ignore);
template <> bool occluded_t<float>(const PhysScene &s, X3<float> o, X3<float> d, float tmax, int ignore) {
	if (g_qc)
		g_qc->any++;
	return occluded(s.bvh, mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), tmax, ignore, g_qc ? &g_qc->ab : nullptr);
}
template <> bool occluded_t<double>(const PhysScene &s, X3<double> o, X3<double> d, double tmax, int ignore) {
	return occluded_d(s, o, d, tmax, ignore);
}

template <typename T> void onb_t(X3<T> n, X3<T> &t, X3<T> &b) {
	T sign = std::copysign(T(1), n.z);
	T a = T(-1) / (sign + n.z);
	T bb = n.x * n.y * a;
	t = x3(T(1) + sign * n.x * n.x * a, sign * bb, -sign * n.x);
	b = x3(bb, sign + n.y * n.y * a, -n.y);
}
template <typename T> T ggx_D_t(T cm, T a2) {
	T k = cm * cm * (a2 - 1) + 1;
	return a2 / (T(3.14159265358979323846) * k * k);
}
template <typename T> T ggx_L_t(T c, T a2) {
	T c2 = c * c;
	T t2 = std::max(T(0), 1 - c2) / std::max(c2, T(1e-12));
	return T(0.5) * (-1 + std::sqrt(1 + a2 * t2));
}
template <typename T> X3<T> schlick_t(X3<T> f0, T c) {
	T m = std::min(std::max(1 - c, T(0)), T(1));
	T m5 = (m * m) * (m * m) * m;
	return f0 + (x3<T>(1, 1, 1) - f0) * m5;
}
template <typename T> T m5_t(T c) {
	T m = std::min(std::max(1 - c, T(0)), T(1));
	return (m * m) * (m * m) * m;
}
template <typename T>
bool eval_t(int mat, X3<T> alb, T alpha, X3<T> n, X3<T> wo, X3<T> wi, X3<T> &fc, T &pdf, T *m5 = nullptr) {
	T ci = dt(n, wi), co = dt(n, wo);
	if (ci <= 0 || co <= 0)
		return false;
	const T inv_pi = T(0.318309886183790671537767526745);
	if (mat == 0) {
		fc = alb * (ci * inv_pi);
		pdf = ci * inv_pi;
		return true;
	}
	T a2 = alpha * alpha;
	X3<T> m = nz(wo + wi);
	T cm = dt(n, m), om = dt(wo, m);
	if (cm <= 0 || om <= 0)
		return false;
	T D = ggx_D_t(cm, a2), lo = ggx_L_t(co, a2), li = ggx_L_t(ci, a2);
	T G2 = 1 / (1 + lo + li), G1 = 1 / (1 + lo);
	fc = schlick_t(alb, om) * (D * G2 / (4 * co));
	pdf = G1 * D / (4 * co);
	if (m5)
		*m5 = m5_t(om);
	return true;
}
template <typename T> T mis_t(T a, T b) { return a * a / (a * a + b * b); }

// d log(weight) / d albedo of a Lambert (1 / albedo) or GGX-Schlick ((1 - m5) / F) vertex.
template <typename T> X3<T> dlog_t(int mat, X3<T> alb, T m5) {
	if (mat == 0)
		return x3<T>(1 / std::max(alb.x, T(1e-12)), 1 / std::max(alb.y, T(1e-12)), 1 / std::max(alb.z, T(1e-12)));
	if (mat == 1) {
		X3<T> F = alb + (x3<T>(1, 1, 1) - alb) * m5;
		T d = 1 - m5;
		return x3<T>(d / std::max(F.x, T(1e-12)), d / std::max(F.y, T(1e-12)), d / std::max(F.z, T(1e-12)));
	}
	return x3<T>(0, 0, 0);
}

// Gradient sink of the replay pass (path replay backpropagation): g = dL/dI / spp,
// C = the path's radiance from the first pass, P = radiance gathered so far.
template <typename T> struct GradSink {
	X3<T> g, C, P;
	double *galb, *gem;
	void add(double *buf, int tri, X3<T> v) {
		double *p = buf + 3 * static_cast<size_t>(tri);
#pragma omp atomic
		p[0] += static_cast<double>(v.x);
#pragma omp atomic
		p[1] += static_cast<double>(v.y);
#pragma omp atomic
		p[2] += static_cast<double>(v.z);
	}
};
template <typename T> X3<T> sdiv(X3<T> a, X3<T> b) {
	return x3<T>(b.x > 0 ? a.x / b.x : T(0), b.y > 0 ? a.y / b.y : T(0), b.z > 0 ? a.z / b.z : T(0));
}

// sin(2 pi u), cos(2 pi u). In double: the C library's. In float: the product's
// quarter-turn reduction and Taylor polynomials (rednoise_b200/csrc/physical.cuh,
// sincos_turn), restated operation by operation so that the FP32 estimator draws the
// same directions bit for bit: u * 4 and the removal of its integer part are exact,
// x = f * pi/2 with |x| <= pi/4, sin to x^11 and cos to x^12 by Horner's rule.
inline void sincos_turn_t(double u, double &s, double &c) {
	const double a = 6.28318530717958647692 * u;
	s = std::sin(a);
	c = std::cos(a);
}
inline void sincos_turn_t(float u, float &s, float &c) {
	const float t = u * 4.0f;
	int q = static_cast<int>(t);
	float f = t - static_cast<float>(q);
	if (f > 0.5f) {
		f = f - 1.0f;
		q = q + 1;
	}
	const float x = f * 1.57079632679489662f;
	const float x2 = x * x;
	const float c11 = -2.50521083854417188e-8f, c9 = 2.75573192239858907e-6f, c7 = -1.98412698412698413e-4f;
	const float c5 = 8.33333333333333333e-3f, c3 = -1.66666666666666667e-1f;
	const float sp = x + x * x2 * (c3 + x2 * (c5 + x2 * (c7 + x2 * (c9 + x2 * c11))));
	const float d12 = 2.08767569878680990e-9f, d10 = -2.75573192239858907e-7f, d8 = 2.48015873015873016e-5f;
	const float d6 = -1.38888888888888889e-3f, d4 = 4.16666666666666667e-2f, d2 = -0.5f;
	const float cp = 1.0f + x2 * (d2 + x2 * (d4 + x2 * (d6 + x2 * (d8 + x2 * (d10 + x2 * d12)))));
	const int k = q & 3;
	s = k == 0 ? sp : k == 1 ? cp : k == 2 ? -sp : -cp;
	c = k == 0 ? cp : k == 1 ? -sp : k == 2 ? -cp : sp;
}

// Continuation sampling of the physical estimator: Lambert (cosine), GGX (visible
// normals, Heitz 2018) or smooth dielectric (Fresnel choice). wi, weight = f cos /
// pdf, pdf (0 for the delta dielectric) and d log(weight) / d albedo; false when the
// sample is absorbed (below the surface).
template <typename T>
bool sample_t(int mat, X3<T> alb, T param, X3<T> n, X3<T> wo, X3<T> d, T cog, T u1, T u2, T uf, X3<T> &wi,
              X3<T> &weight, T &pdf, X3<T> &cont_dlog) {
	cont_dlog = x3<T>(0, 0, 0);
	pdf = 0;
	if (mat == 0) {
		T r = std::sqrt(u1);
		T sn, cs;
		sincos_turn_t(u2, sn, cs);
		X3<T> t, bt;
		onb_t(n, t, bt);
		T z = std::sqrt(std::max(T(0), 1 - u1));
		wi = t * (r * cs) + bt * (r * sn) + n * z;
		T ci = dt(wi, n);
		if (ci <= 0)
			return false;
		weight = alb;
		pdf = ci * T(0.318309886183790671537767526745);
		cont_dlog = dlog_t(0, alb, T(0));
	} else if (mat == 1) {
		T alpha = param, a2 = alpha * alpha;
		X3<T> t, bt;
		onb_t(n, t, bt);
		X3<T> wl = x3(dt(wo, t), dt(wo, bt), dt(wo, n));
		X3<T> vh = nz(x3(alpha * wl.x, alpha * wl.y, wl.z));
		T lensq = vh.x * vh.x + vh.y * vh.y;
		X3<T> T1 = lensq > 0 ? x3<T>(-vh.y, vh.x, 0) * (T(1) / std::sqrt(lensq)) : x3<T>(1, 0, 0);
		X3<T> T2 = cr(vh, T1);
		T r = std::sqrt(u1);
		T sn, cs;
		sincos_turn_t(u2, sn, cs);
		T t1 = r * cs, t2 = r * sn;
		T sb = T(0.5) * (1 + vh.z);
		t2 = (1 - sb) * std::sqrt(std::max(T(0), 1 - t1 * t1)) + sb * t2;
		X3<T> nh = T1 * t1 + T2 * t2 + vh * std::sqrt(std::max(T(0), 1 - t1 * t1 - t2 * t2));
		X3<T> ml = nz(x3(alpha * nh.x, alpha * nh.y, std::max(T(0), nh.z)));
		X3<T> m = t * ml.x + bt * ml.y + n * ml.z;
		T om = dt(wo, m);
		wi = m * (2 * om) - wo;
		T ci = dt(wi, n), co = wl.z;
		if (ci <= 0 || om <= 0 || co <= 0)
			return false;
		T lo_ = ggx_L_t(co, a2), li_ = ggx_L_t(ci, a2);
		T G1 = 1 / (1 + lo_), G2 = 1 / (1 + lo_ + li_);
		weight = schlick_t(alb, om) * (G2 / G1);
		pdf = G1 * ggx_D_t(ml.z, a2) / (4 * co);
		cont_dlog = dlog_t(1, alb, m5_t(om));
	} else {
		T eta = param;
		bool entering = cog > 0;
		T ei = entering ? T(1) : eta, et = entering ? eta : T(1);
		T ci = std::fabs(cog), rel = ei / et;
		T s2t = rel * rel * std::max(T(0), 1 - ci * ci);
		T F = 1, ct = 0;
		if (s2t < 1) {
			ct = std::sqrt(1 - s2t);
			T rs = (ei * ci - et * ct) / (ei * ci + et * ct), rp = (et * ci - ei * ct) / (et * ci + ei * ct);
			F = T(0.5) * (rs * rs + rp * rp);
		}
		if (uf < F)
			wi = n * (2 * ci) - wo;
		else
			wi = d * rel + n * (rel * ci - ct);
		weight = x3<T>(1, 1, 1);
		pdf = 0;
	}
	return true;
}

template <typename T>
X3<T> trace_phys(const PhysScene &s, const PhysCam &c, const PhysSet &st, uint32_t pix, uint32_t sample,
                 GradSink<T> *gs = nullptr) {
	orc::U4 r0 = prand(st.seed, pix, sample, 0);
	int px = static_cast<int>(pix % static_cast<uint32_t>(c.w)), py = static_cast<int>(pix / static_cast<uint32_t>(c.w));
	T sx = ((T(px) + T(orc::u01(r0.x))) / T(c.w)) * 2 - 1;
	T sy = 1 - ((T(py) + T(orc::u01(r0.y))) / T(c.h)) * 2;
	X3<T> fwd = x3<T>(c.fwd[0], c.fwd[1], c.fwd[2]), right = x3<T>(c.right[0], c.right[1], c.right[2]),
	      up = x3<T>(c.up[0], c.up[1], c.up[2]);
	X3<T> o = x3<T>(c.pos[0], c.pos[1], c.pos[2]);
	X3<T> d = nz(fwd + right * (sx * T(c.tan_half) * T(c.aspect)) + up * (sy * T(c.tan_half)));
	X3<T> beta = x3<T>(1, 1, 1), L = x3<T>(0, 0, 0);
	T prev_pdf = 0;
	int ignore = -1;
	const T eps = T(2e-4);
	for (int bounce = 0;; bounce++) {
		PHit<T> h = closest_t<T>(s, o, d, ignore);
		if (h.idx < 0) {
			L = L + beta * x3<T>(st.env[0], st.env[1], st.env[2]);
			break;
		}
		size_t k = static_cast<size_t>(h.idx);
		X3<T> ng = x3<T>(s.normal[3 * k], s.normal[3 * k + 1], s.normal[3 * k + 2]);
		X3<T> p = o + d * h.t;
		X3<T> wo = -d;
		T cog = dt(ng, wo);
		X3<T> Le = x3<T>(s.emission[3 * k], s.emission[3 * k + 1], s.emission[3 * k + 2]);
		if (Le.x > 0 || Le.y > 0 || Le.z > 0) {
			if (cog > 0) {
				T w = 1;
				if (prev_pdf > 0)
					w = mis_t(prev_pdf, h.t * h.t / (cog * T(s.area_total)));
				X3<T> e = beta * Le * w;
				L = L + e;
				if (gs) {
					gs->P = gs->P + e;
					gs->add(gs->gem, h.idx, gs->g * sdiv(e, Le));
				}
			}
			break;
		}
		int mat = s.material[k];
		X3<T> alb = x3<T>(s.albedo[3 * k], s.albedo[3 * k + 1], s.albedo[3 * k + 2]);
		T param = s.param[k];
		X3<T> n = cog >= 0 ? ng : -ng;
		uint32_t b = static_cast<uint32_t>(bounce);
		orc::U4 rA = prand(st.seed, pix, sample, 2u + 2u * b), rB = prand(st.seed, pix, sample, 3u + 2u * b);
		if (mat != 2 && !s.em.empty()) {
			float target = orc::u01(rA.x) * s.area_total;
			int lo = 0, hi = static_cast<int>(s.em.size()) - 1;
			while (lo < hi) {
				int mid = (lo + hi) >> 1;
				if (s.em[mid].cdf > target)
					hi = mid;
				else
					lo = mid + 1;
			}
			const PhysScene::Em &E = s.em[lo];
			T su = std::sqrt(T(orc::u01(rA.y)));
			T b1 = T(orc::u01(rA.z)) * su, b2 = 1 - su;
			X3<T> q = x3<T>(E.v0[0], E.v0[1], E.v0[2]) + x3<T>(E.e0[0], E.e0[1], E.e0[2]) * b1 +
			          x3<T>(E.e1[0], E.e1[1], E.e1[2]) * b2;
			X3<T> wi = q - p;
			T dist2 = dt(wi, wi), dist = std::sqrt(dist2);
			wi = wi * (T(1) / dist);
			size_t ek = static_cast<size_t>(E.tri);
			X3<T> ne = x3<T>(s.normal[3 * ek], s.normal[3 * ek + 1], s.normal[3 * ek + 2]);
			T cos_l = -dt(ne, wi);
			X3<T> fc;
			T pb;
			T m5l = 0;
			if (cos_l > 0 && dist > 0 && eval_t<T>(mat, alb, param, n, wo, wi, fc, pb, &m5l)) {
				T pl = dist2 / (cos_l * T(s.area_total));
				X3<T> eLe = x3<T>(s.emission[3 * ek], s.emission[3 * ek + 1], s.emission[3 * ek + 2]);
				T w = mis_t(pl, pb);
				if (!occluded_t<T>(s, p + n * eps, wi, dist, E.tri)) {
					X3<T> nee = beta * fc * eLe * (w / pl);
					L = L + nee;
					if (gs) {
						gs->P = gs->P + nee;
						gs->add(gs->galb, h.idx, gs->g * nee * dlog_t(mat, alb, m5l));
						gs->add(gs->gem, E.tri, gs->g * sdiv(nee, eLe));
					}
				}
			}
		}
		if (bounce + 1 >= st.max_depth)
			break;
		X3<T> wi, weight, cont_dlog;
		T pdf = 0;
		if (!sample_t<T>(mat, alb, param, n, wo, d, cog, T(orc::u01(rB.x)), T(orc::u01(rB.y)), T(orc::u01(rA.w)), wi,
		                 weight, pdf, cont_dlog))
			break;
		beta = beta * weight;
		if (bounce + 1 >= st.rr_depth) {
			T q = std::min(T(0.95), mx(beta));
			if (!(T(orc::u01(rB.z)) < q))
				break;
			beta = beta * (T(1) / q);
		}
		if (gs)
			gs->add(gs->galb, h.idx, gs->g * (gs->C - gs->P) * cont_dlog);
		T side = dt(wi, ng) >= 0 ? T(1) : T(-1);
		o = p + ng * (side * eps);
		d = wi;
		prev_pdf = pdf;
		ignore = h.idx;
	}
	return L;
}

} // namespace

extern "C" {

// ---- BVH ---------------------------------------------------------------------------

void *orc_bvh_new(int n, const float *v9) {
	Bvh *b = new Bvh();
	b->tris.resize(static_cast<size_t>(n));
	b->cent.resize(static_cast<size_t>(n));
	b->order.resize(static_cast<size_t>(n));
	for (int i = 0; i < n; i++) {
		const float *p = v9 + 9 * static_cast<size_t>(i);
		b->tris[i] = {mk(p[0], p[1], p[2]), mk(p[3], p[4], p[5]), mk(p[6], p[7], p[8])};
		b->cent[i] = (b->tris[i].v0 + b->tris[i].v1 + b->tris[i].v2) / 3.0f;
		b->order[i] = i;
	}
	if (n > 0)
		b->root = b->build(0, n);
	return b;
}

void orc_bvh_free(void *h) { delete static_cast<Bvh *>(h); }

int orc_bvh_node_count(const void *h) { return static_cast<int>(static_cast<const Bvh *>(h)->nodes.size()); }

void orc_bvh_dump(const void *h, int *order, float *bounds, int *links) {
	const Bvh *b = static_cast<const Bvh *>(h);
	std::memcpy(order, b->order.data(), b->order.size() * sizeof(int));
	for (size_t i = 0; i < b->nodes.size(); i++) {
		const Node &n = b->nodes[i];
		const float bb[6] = {n.bmin.x, n.bmin.y, n.bmin.z, n.bmax.x, n.bmax.y, n.bmax.z};
		std::memcpy(bounds + 6 * i, bb, sizeof(bb));
		links[4 * i] = n.left;
		links[4 * i + 1] = n.right;
		links[4 * i + 2] = n.start;
		links[4 * i + 3] = n.count;
	}
}

// Closest hit; boxes/tris (optional) receive the per-ray box and triangle test counts.
void orc_intersect(const void *h, int n, const float *o3, const float *d3, const int *ignore, int *idx, float *t,
                   float *u, float *v, int *boxes, int *tris) {
	const Bvh *b = static_cast<const Bvh *>(h);
#pragma omp parallel for schedule(dynamic, 256)
	for (int i = 0; i < n; i++) {
		Counts c;
		Hit r = intersect(*b, mk(o3[3 * i], o3[3 * i + 1], o3[3 * i + 2]), mk(d3[3 * i], d3[3 * i + 1], d3[3 * i + 2]),
		                  ignore ? ignore[i] : -1, &c);
		idx[i] = r.hit ? r.idx : -1;
		t[i] = r.t;
		u[i] = r.u;
		v[i] = r.v;
		if (boxes)
			boxes[i] = static_cast<int>(c.boxes);
		if (tris)
			tris[i] = static_cast<int>(c.tris);
	}
}

void orc_occluded(const void *h, int n, const float *o3, const float *d3, const float *maxd, const int *ignore,
                  int *occ, int *boxes, int *tris) {
	const Bvh *b = static_cast<const Bvh *>(h);
#pragma omp parallel for schedule(dynamic, 256)
	for (int i = 0; i < n; i++) {
		Counts c;
		occ[i] = occluded(*b, mk(o3[3 * i], o3[3 * i + 1], o3[3 * i + 2]), mk(d3[3 * i], d3[3 * i + 1], d3[3 * i + 2]),
		                  maxd[i], ignore ? ignore[i] : -1, &c)
		             ? 1
		             : 0;
		if (boxes)
			boxes[i] = static_cast<int>(c.boxes);
		if (tris)
			tris[i] = static_cast<int>(c.tris);
	}
}

// ---- reference-mode render -----------------------------------------------------
// Lights: 24-float records [type, pos3, dir3, colour3, I, radius, coneCos, kc, kl, kq, u3, v3, pad2];
// n_lights == 0 -> the reference's default light (0.15 disk at (0, 0.95, 0)).
// Renders rows [y0, y1) of a w x h image with the camera of Camera(w, h, focal, pos) + lookAt(target),
// scale 150; writes argb (w x (y1-y0)) and optionally mean (3 floats per pixel).
void orc_render_reference(const void *bvh, const float *normal3, const int *material, const int *rgb,
                          const float *roughness, int w, int h, int y0, int y1, float focal, const float *pos3,
                          const float *target3, int samples, int max_depth, int n_lights, const float *lights,
                          uint32_t *argb, float *mean) {
	const Bvh *b = static_cast<const Bvh *>(bvh);
	RefScene s;
	s.bvh = b;
	s.max_depth = max_depth;
	const size_t n = b->tris.size();
	s.tri.resize(n);
	for (size_t i = 0; i < n; i++) {
		s.tri[i].normal = mk(normal3[3 * i], normal3[3 * i + 1], normal3[3 * i + 2]);
		s.tri[i].material = material[i];
		s.tri[i].rgb = mk(static_cast<float>(rgb[3 * i]), static_cast<float>(rgb[3 * i + 1]),
		                  static_cast<float>(rgb[3 * i + 2]));
		s.tri[i].roughness = roughness[i];
	}
	if (n_lights == 0) {
		Light d{};
		d.type = kPoint;
		d.pos = mk(0.0f, 0.95f, 0.0f);
		d.dir = mk(0.0f, -1.0f, 0.0f);
		d.colour = mk(1, 1, 1);
		d.intensity = 40.0f;
		d.radius = 0.15f;
		d.cone_cos = 0.9f;
		d.kc = 0.0f;
		d.kl = 0.0f;
		d.kq = 12.566370f;
		d.u = mk(0.3f, 0, 0);
		d.v = mk(0, 0, 0.3f);
		s.lights.push_back(d);
	}
	for (int i = 0; i < n_lights; i++) {
		const float *r = lights + 24 * static_cast<size_t>(i);
		Light L;
		L.type = static_cast<int>(r[0]);
		L.pos = mk(r[1], r[2], r[3]);
		L.dir = mk(r[4], r[5], r[6]);
		L.colour = mk(r[7], r[8], r[9]);
		L.intensity = r[10];
		L.radius = r[11];
		L.cone_cos = r[12];
		L.kc = r[13];
		L.kl = r[14];
		L.kq = r[15];
		L.u = mk(r[16], r[17], r[18]);
		L.v = mk(r[19], r[20], r[21]);
		s.lights.push_back(L);
	}
	V3 pos = mk(pos3[0], pos3[1], pos3[2]), tgt = mk(target3[0], target3[1], target3[2]);
	V3 fwd = normalize(pos - tgt);
	V3 right = normalize(cross(mk(0, 1, 0), fwd));
	V3 up = cross(fwd, right);
	float f = focal * 150.0f;
#pragma omp parallel for schedule(dynamic, 1)
	for (int y = y0; y < y1; y++) {
		for (int x = 0; x < w; x++) {
			Rng rng(static_cast<unsigned>((static_cast<unsigned>(y) * static_cast<unsigned>(w) +
			                               static_cast<unsigned>(x)) *
			                                  9781u +
			                              1u));
			std::uniform_real_distribution<float> jit(-0.5f, 0.5f);
			V3 sum = mk(0, 0, 0);
			for (int sidx = 0; sidx < samples; sidx++) {
				float jx = jit(rng), jy = jit(rng);
				float sx = x + 0.5f + jx - w / 2.0f, sy = -(y + 0.5f + jy - h / 2.0f);
				V3 vv = mk(sx / f, sy / f, -1.0f);
				V3 dir = normalize(right * vv.x + up * vv.y + fwd * vv.z);
				(void)U01(rng); // the motion-blur draw the reference always makes
				sum = sum + path_trace(s, pos, dir, max_depth, rng);
			}
			V3 c = sum / static_cast<float>(samples) * 255.0f;
			auto cv = [](float v) {
				return (v >= -2147483648.0f && v < 2147483648.0f) ? static_cast<int>(v)
				                                                   : static_cast<int>(0x80000000u);
			};
			int r = std::min(255, cv(c.x)), g = std::min(255, cv(c.y)), bl = std::min(255, cv(c.z));
			size_t k = static_cast<size_t>(y - y0) * static_cast<size_t>(w) + static_cast<size_t>(x);
			argb[k] = (255u << 24) | ((static_cast<uint32_t>(r) & 0xFF) << 16) |
			          ((static_cast<uint32_t>(g) & 0xFF) << 8) | (static_cast<uint32_t>(bl) & 0xFF);
			if (mean) {
				V3 m = sum / static_cast<float>(samples);
				mean[3 * k] = m.x;
				mean[3 * k + 1] = m.y;
				mean[3 * k + 2] = m.z;
			}
		}
	}
}

// ---- physical mode ---------------------------------------------------------------

void *orc_pt_scene_new(int n, const float *v9, const float *albedo, const float *emission, const int *material,
                       const float *param) {
	PhysScene *s = new PhysScene();
	Bvh &b = s->bvh;
	b.tris.resize(static_cast<size_t>(n));
	b.cent.resize(static_cast<size_t>(n));
	b.order.resize(static_cast<size_t>(n));
	s->normal.resize(3 * static_cast<size_t>(n));
	double acc = 0.0;
	for (int i = 0; i < n; i++) {
		const float *p = v9 + 9 * static_cast<size_t>(i);
		b.tris[i] = {mk(p[0], p[1], p[2]), mk(p[3], p[4], p[5]), mk(p[6], p[7], p[8])};
		b.cent[i] = (b.tris[i].v0 + b.tris[i].v1 + b.tris[i].v2) / 3.0f;
		b.order[i] = i;
		double ax = double(p[3]) - p[0], ay = double(p[4]) - p[1], az = double(p[5]) - p[2];
		double bx = double(p[6]) - p[0], by = double(p[7]) - p[1], bz = double(p[8]) - p[2];
		double cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
		double len = std::sqrt(cx * cx + cy * cy + cz * cz);
		for (int a = 0; a < 3; a++)
			s->normal[3 * i + a] = len > 0 ? static_cast<float>((a == 0 ? cx : a == 1 ? cy : cz) / len) : 0.0f;
		const float *e = emission + 3 * static_cast<size_t>(i);
		if ((e[0] > 0 || e[1] > 0 || e[2] > 0) && 0.5 * len > 0) {
			acc += 0.5 * len;
			PhysScene::Em E;
			for (int a = 0; a < 3; a++) {
				E.v0[a] = p[a];
				E.e0[a] = p[3 + a] - p[a];
				E.e1[a] = p[6 + a] - p[a];
			}
			E.area = static_cast<float>(0.5 * len);
			E.cdf = static_cast<float>(acc);
			E.tri = i;
			s->em.push_back(E);
		}
	}
	s->area_total = static_cast<float>(acc);
	if (n > 0)
		b.root = b.build(0, n);
	s->albedo.assign(albedo, albedo + 3 * static_cast<size_t>(n));
	s->emission.assign(emission, emission + 3 * static_cast<size_t>(n));
	s->material.assign(material, material + n);
	s->param.assign(param, param + n);
	return s;
}

void orc_pt_scene_free(void *h) { delete static_cast<PhysScene *>(h); }

// Count the reference-order ray queries of the FP32 estimator on the listed
// pixels: out[0..5] = closest queries, any-hit queries, closest box tests,
// closest triangle tests, any-hit box tests, any-hit triangle tests.
void orc_pt_count(const void *h, const float *cam10, int w, int hgt, int spp, int max_depth, int rr_depth,
                  unsigned long long seed, unsigned offset, const float *env3, int n_pix, const int *pixels,
                  long long *out);

// Camera basis as the product's host code builds it (double, rounded once).
static PhysCam make_cam(const float *cam10, int w, int hgt) {
	PhysCam c;
	double pos[3], fwd[3], up[3], right[3], upv[3];
	for (int a = 0; a < 3; a++) {
		pos[a] = cam10[a];
		fwd[a] = double(cam10[3 + a]) - cam10[a];
		up[a] = cam10[6 + a];
	}
	auto nrm = [](double v[3]) {
		double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
		for (int a = 0; a < 3; a++)
			v[a] /= l;
	};
	auto crs = [](const double a[3], const double b[3], double o[3]) {
		o[0] = a[1] * b[2] - a[2] * b[1];
		o[1] = a[2] * b[0] - a[0] * b[2];
		o[2] = a[0] * b[1] - a[1] * b[0];
	};
	nrm(fwd);
	crs(fwd, up, right);
	nrm(right);
	crs(right, fwd, upv);
	for (int a = 0; a < 3; a++) {
		c.pos[a] = float(pos[a]);
		c.fwd[a] = float(fwd[a]);
		c.right[a] = float(right[a]);
		c.up[a] = float(upv[a]);
	}
	c.tan_half = float(std::tan(cam10[9] * 3.14159265358979323846 / 360.0));
	c.aspect = float(w) / float(hgt);
	c.w = w;
	c.h = hgt;
	return c;
}

void orc_pt_count(const void *h, const float *cam10, int w, int hgt, int spp, int max_depth, int rr_depth,
                  unsigned long long seed, unsigned offset, const float *env3, int n_pix, const int *pixels,
                  long long *out) {
	const PhysScene &s = *static_cast<const PhysScene *>(h);
	const PhysCam c = make_cam(cam10, w, hgt);
	PhysSet st{spp, max_depth, rr_depth, seed, offset, {env3[0], env3[1], env3[2]}};
	const int count = pixels ? n_pix : w * hgt;
	long long tot[6] = {0, 0, 0, 0, 0, 0};
#pragma omp parallel
	{
		QueryCounts qc;
		g_qc = &qc;
#pragma omp for schedule(dynamic, 16)
		for (int i = 0; i < count; i++) {
			uint32_t pix = static_cast<uint32_t>(pixels ? pixels[i] : i);
			for (int k = 0; k < spp; k++)
				(void)trace_phys<float>(s, c, st, pix, offset + static_cast<uint32_t>(k));
		}
		g_qc = nullptr;
#pragma omp critical
		{
			tot[0] += qc.closest;
			tot[1] += qc.any;
			tot[2] += qc.cb.boxes;
			tot[3] += qc.cb.tris;
			tot[4] += qc.ab.boxes;
			tot[5] += qc.ab.tris;
		}
	}
	for (int k = 0; k < 6; k++)
		out[k] = tot[k];
}

// Path-replay gradient of the estimator: dimg = dL/d(mean image) (w*h*3 floats),
// galb / gem receive dL/d albedo and dL/d emission (n*3 doubles, overwritten).
// Each sample is traced once for its radiance and once more to scatter derivatives.
void orc_pt_backward(const void *h, const float *cam10, int w, int hgt, int spp, int max_depth, int rr_depth,
                     unsigned long long seed, unsigned offset, const float *env3, const float *dimg, int precision,
                     double *galb, double *gem) {
	const PhysScene &s = *static_cast<const PhysScene *>(h);
	const PhysCam c = make_cam(cam10, w, hgt);
	PhysSet st{spp, max_depth, rr_depth, seed, offset, {env3[0], env3[1], env3[2]}};
	const size_t n = s.bvh.tris.size();
	std::fill(galb, galb + 3 * n, 0.0);
	std::fill(gem, gem + 3 * n, 0.0);
	const int count = w * hgt;
#pragma omp parallel for schedule(dynamic, 16)
	for (int i = 0; i < count; i++) {
		const double inv = spp > 0 ? 1.0 / spp : 0.0;
		for (int k = 0; k < spp; k++) {
			const uint32_t smp = offset + static_cast<uint32_t>(k);
			if (precision == 0) {
				GradSink<float> gs;
				gs.g = x3<float>(float(dimg[3 * i] * inv), float(dimg[3 * i + 1] * inv), float(dimg[3 * i + 2] * inv));
				gs.C = trace_phys<float>(s, c, st, static_cast<uint32_t>(i), smp);
				gs.P = x3<float>(0, 0, 0);
				gs.galb = galb;
				gs.gem = gem;
				(void)trace_phys<float>(s, c, st, static_cast<uint32_t>(i), smp, &gs);
			} else {
				GradSink<double> gs;
				gs.g = x3<double>(dimg[3 * i] * inv, dimg[3 * i + 1] * inv, dimg[3 * i + 2] * inv);
				gs.C = trace_phys<double>(s, c, st, static_cast<uint32_t>(i), smp);
				gs.P = x3<double>(0, 0, 0);
				gs.galb = galb;
				gs.gem = gem;
				(void)trace_phys<double>(s, c, st, static_cast<uint32_t>(i), smp, &gs);
			}
		}
	}
}

// cam: pos3, target3, up3, vfov_deg (10 floats), w, h; settings: spp, max_depth, rr_depth, seed, offset, env3.
// Renders the listed pixels (or all when pixels == NULL) and writes per-pixel SUMS (3 doubles each).
void orc_pt_render(const void *h, const float *cam10, int w, int hgt, int spp, int max_depth, int rr_depth,
                   unsigned long long seed, unsigned offset, const float *env3, int n_pix, const int *pixels,
                   int precision, double *sums) {
	const PhysScene &s = *static_cast<const PhysScene *>(h);
	const PhysCam c = make_cam(cam10, w, hgt);
	PhysSet st{spp, max_depth, rr_depth, seed, offset, {env3[0], env3[1], env3[2]}};
	const int count = pixels ? n_pix : w * hgt;
#pragma omp parallel for schedule(dynamic, 16)
	for (int i = 0; i < count; i++) {
		uint32_t pix = static_cast<uint32_t>(pixels ? pixels[i] : i);
		double sx = 0, sy = 0, sz = 0;
		for (int k = 0; k < spp; k++) {
			if (precision == 0) {
				X3<float> L = trace_phys<float>(s, c, st, pix, offset + static_cast<uint32_t>(k));
				sx += L.x;
				sy += L.y;
				sz += L.z;
			} else {
				X3<double> L = trace_phys<double>(s, c, st, pix, offset + static_cast<uint32_t>(k));
				sx += L.x;
				sy += L.y;
				sz += L.z;
			}
		}
		sums[3 * i] = sx;
		sums[3 * i + 1] = sy;
		sums[3 * i + 2] = sz;
	}
}

} // extern "C"

// ---- bidirectional path tracing and PSSMLT ---------------------------------------
// Restated from src/BDPT.cpp:8-144 and src/Metropolis.cpp:8-192: diffuse-only
// estimators lit by the fixed 0.36 x 0.36 ceiling patch at (0, 0.33, 0) facing -y,
// Le = 30. Two random sources drive the bidirectional estimator:
//   * stream 0: the reference's own -- std::mt19937(9871 + y) per image row, drawn
//     through uniform_real_distribution<float>, in the reference's draw order;
//   * stream 1: counter-based -- Philox-4x32-10 keyed by the seed, counter
//     (pixel, sample, block, 0), each 32-bit word mapped as the reference maps an
//     engine output (float(x) / 2^32, clamped below 1).
// The Metropolis sampler restates the reference's mutation and deposition rules
// for the many-chain GPU scheme: chains start from bootstrap paths drawn with
// probability proportional to luminance, and every random number comes from a
// Philox stream (see orc_mlt_render).
// rtl != 0 evaluates the two random arguments of one glm::vec3 constructor or
// cosineHemisphere call right to left, as GCC's x86-64 code does.
namespace {

const float kGiPi = 3.14159265f;
const float kGiEps = 1e-3f;
const float kGiLightHalf = 0.18f;
const float kGiLightArea = (2.0f * kGiLightHalf) * (2.0f * kGiLightHalf);
const float kGiLe = 30.0f;
const int kGiMaxDepth = 4;
const int kMltMaxDims = 2 + 4 * kGiMaxDepth;

struct GiScene {
	const Bvh *bvh;
	std::vector<V3> normal;
	std::vector<V3> albedo; // vec3(colour) / 255
};

struct GiCam {
	V3 pos, right, up, fwd;
	float f;
};

GiCam gi_cam(float focal, const float *pos3, const float *target3) {
	GiCam c;
	c.pos = mk(pos3[0], pos3[1], pos3[2]);
	V3 tgt = mk(target3[0], target3[1], target3[2]);
	c.fwd = normalize(c.pos - tgt);
	c.right = normalize(cross(mk(0, 1, 0), c.fwd));
	c.up = cross(c.fwd, c.right);
	c.f = focal * 150.0f;
	return c;
}

// faceViewer (src/BDPT.cpp:34-36, src/Metropolis.cpp:38-40)
V3 gi_face(V3 n, V3 d) { return dot(n, d) < 0.0f ? n : -n; }

// cosineHemisphere on two given uniforms (src/Metropolis.cpp:42-50)
V3 gi_cosine(V3 n, float u1, float u2) {
	float r = std::sqrt(u1), th = 2.0f * kGiPi * u2;
	float x = r * std::cos(th), y = r * std::sin(th), z = std::sqrt(std::max(0.0f, 1.0f - u1));
	V3 up = std::fabs(n.z) < 0.99f ? mk(0, 0, 1) : mk(1, 0, 0);
	V3 t = normalize(cross(up, n)), b = cross(n, t);
	return normalize(t * x + b * y + n * z);
}

// one engine word -> uniform_real_distribution<float>(0, 1)
float gi_canon(uint32_t x) {
	float c = static_cast<float>(x) / 4294967296.0f;
	if (c >= 1.0f)
		c = std::nextafter(1.0f, 0.0f);
	return c * (1.0f - 0.0f) + 0.0f;
}

uint32_t u4_word(orc::U4 v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }

struct MtDraw {
	Rng rng;
	explicit MtDraw(uint32_t s) : rng(s) {}
	float operator()() { return U01(rng); }
};

// Philox words of counter (a, b, block, tag) under the key (seed), consumed in order.
struct CtrDraw {
	uint32_t a, b, tag, k0, k1;
	int n = 0;
	orc::U4 blk{};
	float operator()() {
		if ((n & 3) == 0)
			blk = orc::philox4x32_10(orc::U4{a, b, static_cast<uint32_t>(n >> 2), tag}, k0, k1);
		return gi_canon(u4_word(blk, n++ & 3));
	}
};

struct GVert {
	V3 p, n, albedo, beta;
	bool light;
};

// tracePath (src/BDPT.cpp:43-61)
template <class D> int gi_subpath(const GiScene &s, V3 o, V3 d, V3 beta, GVert *out, D &draw) {
	int k = 0;
	for (int depth = 0; depth < kGiMaxDepth; depth++) {
		Hit h = intersect(*s.bvh, o, d, -1, nullptr);
		if (!h.hit)
			return k;
		GVert v;
		v.p = h.point;
		v.n = gi_face(s.normal[h.idx], d);
		v.albedo = s.albedo[h.idx];
		v.beta = beta;
		v.light = false;
		out[k++] = v;
		float u1 = draw(), u2 = draw();
		V3 nd = gi_cosine(v.n, u1, u2);
		beta = beta * v.albedo;
		o = v.p + kGiEps * nd;
		d = nd;
	}
	return k;
}

// One sample of renderBidirectional's pixel loop (src/BDPT.cpp:89-134), added to acc.
template <class D>
void bdpt_sample(const GiScene &s, const GiCam &c, int x, int y, int W, int H, D &draw, bool rtl, V3 &acc) {
	float a0 = draw(), a1 = draw();
	float ux = rtl ? a1 : a0, uy = rtl ? a0 : a1;
	V3 dc = mk((static_cast<float>(x) + ux - static_cast<float>(W) / 2.0f) / c.f,
	           -(static_cast<float>(y) + uy - static_cast<float>(H) / 2.0f) / c.f, -1.0f);
	V3 dir = normalize(c.right * dc.x + c.up * dc.y + c.fwd * dc.z);
	GVert cam[kGiMaxDepth];
	int nc = gi_subpath(s, c.pos, dir, mk(1, 1, 1), cam, draw);
	float b0 = draw(), b1 = draw();
	float lx = rtl ? b1 : b0, lz = rtl ? b0 : b1;
	V3 lp = mk(0.0f, 0.33f, 0.0f) + mk((lx * 2.0f - 1.0f) * kGiLightHalf, 0.0f, (lz * 2.0f - 1.0f) * kGiLightHalf);
	const V3 ln = mk(0.0f, -1.0f, 0.0f);
	const V3 le = mk(kGiLe, kGiLe, kGiLe) * kGiLightArea;
	GVert lv[kGiMaxDepth + 1];
	lv[0] = GVert{lp, ln, mk(0, 0, 0), le, true};
	float d1 = draw(), d2 = draw();
	V3 ldir = gi_cosine(ln, d1, d2);
	int nl = 1 + gi_subpath(s, lp + kGiEps * ldir, ldir, le, lv + 1, draw);
	for (int i = 0; i < nc; i++) {
		const GVert &cv = cam[i];
		for (int j = 0; j < nl; j++) {
			const GVert &l = lv[j];
			V3 d = l.p - cv.p;
			float dist2 = dot(d, d);
			float dist = std::sqrt(dist2);
			d = d / dist;
			float cosC = dot(cv.n, d);
			float cosL = dot(l.n, -d);
			if (cosC <= 0.0f || cosL <= 0.0f)
				continue;
			if (occluded(*s.bvh, cv.p + cv.n * kGiEps, d, dist - 2.0f * kGiEps, -1, nullptr))
				continue;
			float G = cosC * cosL / dist2;
			V3 fC = cv.albedo / kGiPi;
			V3 contrib = cv.beta * fC * G * l.beta;
			if (!l.light)
				contrib = contrib * (l.albedo / kGiPi);
			float w = 1.0f / static_cast<float>(i + j + 2);
			acc = acc + contrib * w;
		}
	}
}

int cvt_i(float v) {
	return (v >= -2147483648.0f && v < 2147483648.0f) ? static_cast<int>(v) : static_cast<int>(0x80000000u);
}

// Reinhard and the 8-bit pack of src/BDPT.cpp:136-141 and src/Metropolis.cpp:184-189.
uint32_t gi_pack(V3 c) {
	c = 255.0f * mk(c.x / (c.x + 1.0f), c.y / (c.y + 1.0f), c.z / (c.z + 1.0f));
	int r = std::min(255, cvt_i(c.x)), g = std::min(255, cvt_i(c.y)), b = std::min(255, cvt_i(c.z));
	return (255u << 24) | ((static_cast<uint32_t>(r) & 0xFF) << 16) | ((static_cast<uint32_t>(g) & 0xFF) << 8) |
	       (static_cast<uint32_t>(b) & 0xFF);
}

float luminance(V3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

// The primary-sample vector of one Metropolis state (src/Metropolis.cpp:26-36):
// coordinates past n are drawn on first use from `ext`.
template <class E> struct MltSampler {
	float *u;
	int *n;
	E &ext;
	int idx = 0;
	float next() {
		if (idx >= *n) {
			u[*n] = ext(idx);
			(*n)++;
		}
		return u[idx++];
	}
};

// tracePath with next-event estimation (src/Metropolis.cpp:53-81)
template <class S> V3 mlt_trace(const GiScene &s, S &smp, V3 o, V3 d, bool rtl) {
	V3 L = mk(0, 0, 0), beta = mk(1, 1, 1);
	const V3 ln = mk(0.0f, -1.0f, 0.0f);
	for (int depth = 0; depth < kGiMaxDepth; depth++) {
		Hit h = intersect(*s.bvh, o, d, -1, nullptr);
		if (!h.hit)
			break;
		V3 n = gi_face(s.normal[h.idx], d);
		V3 albedo = s.albedo[h.idx];
		V3 point = h.point;
		float a0 = smp.next(), a1 = smp.next();
		float ux = rtl ? a1 : a0, uz = rtl ? a0 : a1;
		V3 lp = mk(0.0f, 0.33f, 0.0f) + mk((ux * 2.0f - 1.0f) * kGiLightHalf, 0.0f, (uz * 2.0f - 1.0f) * kGiLightHalf);
		V3 toL = lp - point;
		float dist = length(toL);
		toL = toL / dist;
		float cosS = dot(n, toL), cosL = dot(ln, -toL);
		if (cosS > 0.0f && cosL > 0.0f && !occluded(*s.bvh, point + n * kGiEps, toL, dist - 2.0f * kGiEps, -1, nullptr)) {
			float G = cosS * cosL / (dist * dist);
			L = L + beta * (albedo / kGiPi) * G * mk(kGiLe, kGiLe, kGiLe) * kGiLightArea;
		}
		float c0 = smp.next(), c1 = smp.next();
		V3 nd = gi_cosine(n, rtl ? c1 : c0, rtl ? c0 : c1);
		beta = beta * albedo;
		o = point + kGiEps * nd;
		d = nd;
	}
	return L;
}

// eval (src/Metropolis.cpp:96-105): pixel from the first two coordinates.
template <class S> V3 mlt_eval(const GiScene &s, const GiCam &c, int W, int H, S &smp, bool rtl, int &pixel) {
	float fx = smp.next(), fy = smp.next();
	int px = std::min(W - 1, static_cast<int>(fx * static_cast<float>(W)));
	int py = std::min(H - 1, static_cast<int>(fy * static_cast<float>(H)));
	pixel = py * W + px;
	V3 dc = mk((static_cast<float>(px) + 0.5f - static_cast<float>(W) / 2.0f) / c.f,
	           -(static_cast<float>(py) + 0.5f - static_cast<float>(H) / 2.0f) / c.f, -1.0f);
	V3 dir = normalize(c.right * dc.x + c.up * dc.y + c.fwd * dc.z);
	return mlt_trace(s, smp, c.pos, dir, rtl);
}

// Standard normal from two uniforms (Box and Muller 1958), evaluated in double.
float gi_normal(float u1, float u2) {
	return static_cast<float>(std::sqrt(-2.0 * std::log(1.0 - static_cast<double>(u1))) *
	                          std::cos(6.283185307179586 * static_cast<double>(u2)));
}

GiScene gi_scene(const void *bvh, const float *normal3, const int *rgb) {
	GiScene s;
	s.bvh = static_cast<const Bvh *>(bvh);
	const size_t n = s.bvh->tris.size();
	s.normal.resize(n);
	s.albedo.resize(n);
	for (size_t i = 0; i < n; i++) {
		s.normal[i] = mk(normal3[3 * i], normal3[3 * i + 1], normal3[3 * i + 2]);
		s.albedo[i] = mk(static_cast<float>(rgb[3 * i]), static_cast<float>(rgb[3 * i + 1]),
		                 static_cast<float>(rgb[3 * i + 2])) /
		              255.0f;
	}
	return s;
}

} // namespace

extern "C" {

// renderBidirectional over rows [y0, y1) of a w x h image; camera as orc_render_reference.
// stream 0: the reference's per-row mt19937 streams; 1: Philox under `seed`.
// argb: w x (y1 - y0); acc (may be null): 3 floats per pixel, accum * (exposure / samples).
void orc_bdpt_render(const void *bvh, const float *normal3, const int *rgb, int w, int h, int y0, int y1, float focal,
                     const float *pos3, const float *target3, int samples, float exposure, int stream,
                     unsigned long long seed, int rtl, uint32_t *argb, float *acc) {
	const GiScene s = gi_scene(bvh, normal3, rgb);
	const GiCam c = gi_cam(focal, pos3, target3);
#pragma omp parallel for schedule(dynamic, 1)
	for (int y = y0; y < y1; y++) {
		MtDraw mt(static_cast<uint32_t>(9871 + y));
		for (int x = 0; x < w; x++) {
			V3 sum = mk(0, 0, 0);
			for (int k = 0; k < samples; k++) {
				if (stream == 0) {
					bdpt_sample(s, c, x, y, w, h, mt, rtl != 0, sum);
				} else {
					CtrDraw d{static_cast<uint32_t>(y * w + x), static_cast<uint32_t>(k), 0u,
					          static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32)};
					bdpt_sample(s, c, x, y, w, h, d, rtl != 0, sum);
				}
			}
			V3 col = sum * (exposure / static_cast<float>(samples));
			size_t i = static_cast<size_t>(y - y0) * static_cast<size_t>(w) + static_cast<size_t>(x);
			argb[i] = gi_pack(col);
			if (acc) {
				acc[3 * i] = col.x;
				acc[3 * i + 1] = col.y;
				acc[3 * i + 2] = col.z;
			}
		}
	}
}

// The many-chain Metropolis sampler of rednoise_b200 (counter-based random numbers):
//  1. bootstrap: `bootstrap` independent paths, path i drawing coordinate m from
//     Philox counter (i, 0, m / 4, 1) word m % 4; their luminances are summed in
//     1024 contiguous segments (double), then segment by segment: total and b.
//  2. chain c starts at the bootstrap path whose inclusive luminance prefix first
//     exceeds xi * total, xi from counter (c, 0, 0, 2) word 0.
//  3. chain c runs mutations / chains steps (one more for c < mutations % chains);
//     step t draws from counter (c, t, k / 4, 3) word k % 4: k = 0 large-step test,
//     1 acceptance test, 2 + 2m and 3 + 2m coordinate m's mutation (a fresh uniform,
//     or Box-Muller for the small step), 40 + m coordinate m's first draw.
// image (w*h*3) receives the deposits (unscaled); b_out the bootstrap mean luminance.
// argb (may be null): the reference's canvas (scale b * w * h / mutations, exposure, Reinhard).
void orc_mlt_render(const void *bvh, const float *normal3, const int *rgb, int w, int h, float focal,
                    const float *pos3, const float *target3, long long mutations, int chains, int bootstrap,
                    unsigned long long seed, float exposure, int rtl, float *image, double *b_out, uint32_t *argb) {
	const GiScene s = gi_scene(bvh, normal3, rgb);
	const GiCam c = gi_cam(focal, pos3, target3);
	const uint32_t k0 = static_cast<uint32_t>(seed), k1 = static_cast<uint32_t>(seed >> 32);
	const bool r = rtl != 0;
	std::vector<float> lum(static_cast<size_t>(bootstrap));
	std::vector<int> len(static_cast<size_t>(bootstrap));
	for (int i = 0; i < bootstrap; i++) {
		float u[kMltMaxDims];
		int n = 0, pix = 0;
		CtrDraw d{static_cast<uint32_t>(i), 0u, 1u, k0, k1};
		auto ext = [&](int) { return d(); };
		MltSampler<decltype(ext)> smp{u, &n, ext};
		lum[i] = luminance(mlt_eval(s, c, w, h, smp, r, pix));
		len[i] = n;
	}
	const int seg = (bootstrap + 1023) / 1024;
	std::vector<double> cdf(static_cast<size_t>(bootstrap));
	double total = 0.0;
	for (int t = 0; t < 1024; t++) {
		double run = total;
		for (int i = t * seg; i < std::min(bootstrap, (t + 1) * seg); i++) {
			run += static_cast<double>(lum[i]);
			cdf[i] = run;
		}
		double part = 0.0;
		for (int i = t * seg; i < std::min(bootstrap, (t + 1) * seg); i++)
			part += static_cast<double>(lum[i]);
		total += part;
	}
	*b_out = total / static_cast<double>(bootstrap);
	std::fill(image, image + 3 * static_cast<size_t>(w) * h, 0.0f);
	if (total > 0.0) {
		const float sigma = 0.02f, p_large = 0.3f;
		for (int ch = 0; ch < chains; ch++) {
			const float xi = gi_canon(orc::philox4x32_10(orc::U4{static_cast<uint32_t>(ch), 0u, 0u, 2u}, k0, k1).x);
			const double target = static_cast<double>(xi) * total;
			int lo = 0, hi = bootstrap - 1;
			while (lo < hi) {
				int mid = (lo + hi) / 2;
				if (cdf[mid] > target)
					hi = mid;
				else
					lo = mid + 1;
			}
			float cur[kMltMaxDims];
			int cn = 0, cur_pix = 0;
			{
				CtrDraw d{static_cast<uint32_t>(lo), 0u, 1u, k0, k1};
				for (int m = 0; m < len[lo]; m++)
					cur[m] = d();
				cn = len[lo];
			}
			auto never = [](int) { return 0.0f; };
			MltSampler<decltype(never)> s0{cur, &cn, never};
			V3 curL = mlt_eval(s, c, w, h, s0, r, cur_pix);
			float curLum = luminance(curL);
			const long long steps = mutations / chains + (ch < mutations % chains ? 1 : 0);
			for (long long t = 0; t < steps; t++) {
				const uint32_t tc = static_cast<uint32_t>(t);
				auto W = [&](int k) {
					orc::U4 v = orc::philox4x32_10(orc::U4{static_cast<uint32_t>(ch), tc, static_cast<uint32_t>(k >> 2), 3u},
					                               k0, k1);
					return gi_canon(u4_word(v, k & 3));
				};
				const bool large = W(0) < p_large;
				float prop[kMltMaxDims];
				int pn = cn;
				for (int m = 0; m < cn; m++) {
					if (large) {
						prop[m] = W(2 + 2 * m);
					} else {
						float v = cur[m] + sigma * gi_normal(W(2 + 2 * m), W(3 + 2 * m));
						v = v - std::floor(v);
						prop[m] = v;
					}
				}
				auto ext = [&](int m) { return W(40 + m); };
				MltSampler<decltype(ext)> sp{prop, &pn, ext};
				int prop_pix = 0;
				V3 propL = mlt_eval(s, c, w, h, sp, r, prop_pix);
				float propLum = luminance(propL);
				float a = (curLum > 0.0f) ? std::min(1.0f, propLum / curLum) : 1.0f;
				if (propLum > 0.0f) {
					V3 dep = propL * (a / propLum);
					image[3 * prop_pix] += dep.x;
					image[3 * prop_pix + 1] += dep.y;
					image[3 * prop_pix + 2] += dep.z;
				}
				if (curLum > 0.0f) {
					V3 dep = curL * ((1.0f - a) / curLum);
					image[3 * cur_pix] += dep.x;
					image[3 * cur_pix + 1] += dep.y;
					image[3 * cur_pix + 2] += dep.z;
				}
				if (W(1) < a) {
					std::memcpy(cur, prop, sizeof(float) * static_cast<size_t>(pn));
					cn = pn;
					cur_pix = prop_pix;
					curL = propL;
					curLum = propLum;
				}
			}
		}
	}
	if (argb) {
		const float b = static_cast<float>(*b_out);
		if (!(b > 0.0f)) {
			std::fill(argb, argb + static_cast<size_t>(w) * h, 0u);
			return;
		}
		const float scale = b * static_cast<float>(w) * static_cast<float>(h) / static_cast<float>(mutations);
		for (size_t i = 0; i < static_cast<size_t>(w) * h; i++) {
			V3 v = mk(image[3 * i], image[3 * i + 1], image[3 * i + 2]) * scale * exposure;
			argb[i] = gi_pack(v);
		}
	}
}

} // extern "C"

extern "C" {

// The physical estimator's BSDFs in double precision, for analytic checks
// (tests/test_oracle.py): material 0 Lambert, 1 GGX (param = alpha, albedo = F0),
// 2 smooth dielectric (param = IOR). ng: the geometric normal; wo: towards the
// viewer. eval: f cos and the sampling pdf of each wi (ok = 0 below either side).
void orc_bsdf_eval(int mat, const double *alb3, double param, const double *ng3, const double *wo3, int count,
                   const double *wi3, double *fc3, double *pdf, int *ok) {
	X3<double> alb = x3(alb3[0], alb3[1], alb3[2]), ng = x3(ng3[0], ng3[1], ng3[2]);
	X3<double> wo = x3(wo3[0], wo3[1], wo3[2]);
	X3<double> n = dt(ng, wo) >= 0 ? ng : -ng;
	for (int i = 0; i < count; i++) {
		X3<double> wi = x3(wi3[3 * i], wi3[3 * i + 1], wi3[3 * i + 2]), fc = x3(0.0, 0.0, 0.0);
		double p = 0;
		ok[i] = eval_t<double>(mat, alb, param, n, wo, wi, fc, p) ? 1 : 0;
		fc3[3 * i] = fc.x;
		fc3[3 * i + 1] = fc.y;
		fc3[3 * i + 2] = fc.z;
		pdf[i] = p;
	}
}

// The FP32 estimator's sin(2 pi u), cos(2 pi u) on count uniforms (accuracy checks).
void orc_sincos_turn(int count, const float *u, float *s, float *c) {
	for (int i = 0; i < count; i++)
		sincos_turn_t(u[i], s[i], c[i]);
}

// count samples from uniforms u (3 per sample: the two direction uniforms and the
// Fresnel choice): wi, weight = f cos / pdf, pdf, ok (0: absorbed).
void orc_bsdf_sample(int mat, const double *alb3, double param, const double *ng3, const double *wo3, int count,
                     const double *u3, double *wi3, double *weight3, double *pdf, int *ok) {
	X3<double> alb = x3(alb3[0], alb3[1], alb3[2]), ng = x3(ng3[0], ng3[1], ng3[2]);
	X3<double> wo = x3(wo3[0], wo3[1], wo3[2]);
	const double cog = dt(ng, wo);
	X3<double> n = cog >= 0 ? ng : -ng;
	for (int i = 0; i < count; i++) {
		X3<double> wi = x3(0.0, 0.0, 0.0), w = x3(0.0, 0.0, 0.0), dl;
		double p = 0;
		const bool good = sample_t<double>(mat, alb, param, n, wo, -wo, cog, u3[3 * i], u3[3 * i + 1],
		                                   u3[3 * i + 2], wi, w, p, dl);
		ok[i] = good ? 1 : 0;
		wi3[3 * i] = wi.x;
		wi3[3 * i + 1] = wi.y;
		wi3[3 * i + 2] = wi.z;
		weight3[3 * i] = w.x;
		weight3[3 * i + 1] = w.y;
		weight3[3 * i + 2] = w.z;
		pdf[i] = p;
	}
}

} // extern "C"
