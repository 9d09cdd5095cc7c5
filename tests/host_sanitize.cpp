// Host-code check run under AddressSanitizer + UndefinedBehaviorSanitizer and
// under ThreadSanitizer (tests/test_host_sanitize.py builds it): the OBJ/MTL
// loader on well-formed and malformed files, the reference-identical BVH build
// (including its threaded top levels) on random, degenerate and coincident
// triangles, and both device-layout flattenings, with the tree invariants checked;
// also the wavefront's first-queue pixel order (a permutation for every frame size).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <random>
#include <string>
#include <vector>

#include "host_scene.hpp"
#include "pixel_tiles.cuh"

using namespace rnb;

static int g_fail = 0;
#define CHECK(c)                                                                                                       \
	do {                                                                                                               \
		if (!(c)) {                                                                                                    \
			std::printf("check failed: %s (line %d)\n", #c, __LINE__);                                                 \
			g_fail = 1;                                                                                                \
		}                                                                                                              \
	} while (0)

static int as_int(float f) {
	int i;
	std::memcpy(&i, &f, 4);
	return i;
}

static void check_tree(const std::vector<float> &v, const Bvh2 &b) {
	const int n = static_cast<int>(v.size() / 9);
	CHECK(static_cast<int>(b.order.size()) == n);
	std::vector<int> seen(static_cast<size_t>(n), 0);
	for (int t : b.order) {
		CHECK(t >= 0 && t < n);
		if (t >= 0 && t < n)
			seen[t]++;
	}
	for (int c : seen)
		CHECK(c == 1);
	if (n == 0) {
		CHECK(b.root == -1);
		return;
	}
	std::vector<int> in_leaf(static_cast<size_t>(n), 0);
	for (const BvhNode &nd : b.nodes) {
		if (nd.count > 0) {
			CHECK(nd.count <= 4 && nd.start >= 0 && nd.start + nd.count <= n);
			for (int i = nd.start; i < nd.start + nd.count && i < n; i++) {
				in_leaf[i]++;
				const float *t = &v[9 * static_cast<size_t>(b.order[i])];
				for (int k = 0; k < 3; k++) {
					CHECK(t[3 * k] >= nd.bmin.x && t[3 * k] <= nd.bmax.x);
					CHECK(t[3 * k + 1] >= nd.bmin.y && t[3 * k + 1] <= nd.bmax.y);
					CHECK(t[3 * k + 2] >= nd.bmin.z && t[3 * k + 2] <= nd.bmax.z);
				}
			}
		} else {
			const int m = static_cast<int>(b.nodes.size());
			CHECK(nd.left > 0 && nd.left < m && nd.right > 0 && nd.right < m);
			if (nd.left > 0 && nd.left < m && nd.right > 0 && nd.right < m)
				for (int ch : {nd.left, nd.right}) {
					const BvhNode &c = b.nodes[ch];
					CHECK(c.bmin.x >= nd.bmin.x && c.bmax.x <= nd.bmax.x);
					CHECK(c.bmin.y >= nd.bmin.y && c.bmax.y <= nd.bmax.y);
					CHECK(c.bmin.z >= nd.bmin.z && c.bmax.z <= nd.bmax.z);
				}
		}
	}
	for (int c : in_leaf)
		CHECK(c == 1);
	CHECK(b.depth >= 1);
}

static void check_layouts(const std::vector<float> &v, const Bvh2 &b) {
	TriangleSet ts;
	ts.v = v;
	const int n = static_cast<int>(v.size() / 9);
	DeviceLayout lay;
	flatten_bvh(ts, b, lay);
	CHECK(lay.tris.size() == 3 * static_cast<size_t>(n));
	for (int i = 0; i < n; i++) {
		const int orig = as_int(lay.tris[3 * static_cast<size_t>(i)].w);
		CHECK(orig >= 0 && orig < n);
	}
	const int internal = lay.internal_count;
	CHECK(lay.nodes.size() == 4 * static_cast<size_t>(internal));
	auto ref_ok = [&](int r, int nodes) {
		if (r >= 0)
			return r < nodes;
		const int start = (~r) >> 3, count = (~r) & 7;
		return count >= 1 && count <= 4 && start >= 0 && start + count <= n;
	};
	for (int i = 0; i < internal; i++) {
		const F4 &r = lay.nodes[4 * static_cast<size_t>(i) + 3];
		CHECK(ref_ok(as_int(r.x), internal) && ref_ok(as_int(r.y), internal));
	}
	DeviceLayout4 l4;
	flatten_bvh4(b, l4);
	CHECK(l4.nodes.size() % 8 == 0);
	const int n4 = static_cast<int>(l4.nodes.size() / 8);
	for (int i = 0; i < n4; i++) {
		const F4 &refs = l4.nodes[8 * static_cast<size_t>(i) + 6];
		const int cnt = as_int(l4.nodes[8 * static_cast<size_t>(i) + 7].x);
		CHECK(cnt >= 2 && cnt <= 4);
		const int rr[4] = {as_int(refs.x), as_int(refs.y), as_int(refs.z), as_int(refs.w)};
		for (int k = 0; k < cnt && k < 4; k++)
			CHECK(ref_ok(rr[k], n4));
	}
	// With every box passing, the 4-wide layout pops the reference's leaves in the
	// reference's own order (right child first), each exactly once.
	std::vector<int> want, got;
	std::vector<int> st{b.root};
	while (!st.empty()) {
		const BvhNode &nd = b.nodes[static_cast<size_t>(st.back())];
		st.pop_back();
		if (nd.count > 0) {
			want.push_back(~((nd.start << 3) | nd.count));
		} else {
			st.push_back(nd.left);
			st.push_back(nd.right);
		}
	}
	st.assign(1, l4.root_ref);
	size_t guard = 0;
	while (!st.empty() && guard++ < 8 * want.size() + 8) {
		const int r = st.back();
		st.pop_back();
		if (r < 0) {
			got.push_back(r);
			continue;
		}
		CHECK(r < n4);
		if (r >= n4)
			break;
		const F4 *o = &l4.nodes[8 * static_cast<size_t>(r)];
		const int cnt = as_int(o[7].x);
		const int rr[4] = {as_int(o[6].x), as_int(o[6].y), as_int(o[6].z), as_int(o[6].w)};
		for (int k = std::min(cnt, 4); k-- > 0;)
			st.push_back(rr[k]);
	}
	CHECK(got == want);
}

// A complete tree of odd height collapses into full 4-wide nodes only, apart from
// the root: 512 triangles in a row give 2^7 leaves of 4 under a tree of height 7,
// and 1 + 2 + 8 + 32 = 43 nodes (a top-down collapse gives 1 + 4 + 16 + 64 = 85,
// the last 64 with two entries).
static void complete_tree_case() {
	std::vector<float> v;
	for (int i = 0; i < 512; i++) {
		const float x = static_cast<float>(i);
		const float t[9] = {x, 0.0f, 0.0f, x + 0.5f, 1.0f, 0.0f, x + 0.25f, 0.0f, 1.0f};
		v.insert(v.end(), t, t + 9);
	}
	Bvh2 b;
	build_reference_bvh(v.data(), 512, b);
	DeviceLayout4 l4;
	flatten_bvh4(b, l4);
	const int n4 = static_cast<int>(l4.nodes.size() / 8);
	int full = 0;
	for (int i = 0; i < n4; i++)
		full += as_int(l4.nodes[8 * static_cast<size_t>(i) + 7].x) == 4;
	CHECK(b.depth == 8);
	CHECK(n4 == 43);
	CHECK(full == 42);
}

// The first closest-hit queue's pixel order is a permutation of the frame's pixels
// for every frame size, whole 8 x 4 tiles or not.
static void tile_order_cases() {
	for (uint32_t w = 1; w <= 41; w++)
		for (uint32_t h = 1; h <= 13; h++) {
			std::vector<int> seen(static_cast<size_t>(w) * h, 0);
			for (uint32_t p = 0; p < w * h; p++) {
				const uint32_t t = tile_order(p, w, h);
				CHECK(t < w * h);
				if (t < w * h)
					seen[t]++;
			}
			for (int c : seen)
				CHECK(c == 1);
		}
	const uint32_t w = 1920, h = 1080;
	std::vector<uint8_t> seen(static_cast<size_t>(w) * h, 0);
	bool ok = true;
	for (uint32_t p = 0; p < w * h; p++) {
		const uint32_t t = tile_order(p, w, h);
		ok = ok && t < w * h && !seen[t];
		if (t < w * h)
			seen[t] = 1;
	}
	CHECK(ok);
	CHECK(tile_order(0, w, h) == 0 && tile_order(1, w, h) == 1 && tile_order(w, w, h) == 8);
}

static void tree_case(const std::vector<float> &v) {
	Bvh2 b;
	build_reference_bvh(v.data(), static_cast<int>(v.size() / 9), b);
	check_tree(v, b);
	if (!v.empty())
		check_layouts(v, b);
}

static std::vector<float> soup(int n, unsigned seed, float scale) {
	std::mt19937 rng(seed);
	std::uniform_real_distribution<float> u(-1.0f, 1.0f);
	std::vector<float> v(9 * static_cast<size_t>(n));
	for (int i = 0; i < n; i++) {
		const float cx = u(rng) * scale, cy = u(rng) * scale, cz = u(rng) * scale;
		for (int k = 0; k < 3; k++) {
			v[9 * static_cast<size_t>(i) + 3 * k] = cx + 0.01f * scale * u(rng);
			v[9 * static_cast<size_t>(i) + 3 * k + 1] = cy + 0.01f * scale * u(rng);
			v[9 * static_cast<size_t>(i) + 3 * k + 2] = cz + 0.01f * scale * u(rng);
		}
	}
	return v;
}

static void write(const std::string &path, const std::string &text) { std::ofstream(path) << text; }

static void loader_cases(const std::string &dir) {
	const std::string mtl = dir + "/m.mtl", obj = dir + "/a.obj";
	write(mtl, "newmtl Red\nKd 1 0 0\nnewmtl Glass\nKd 0.5 0.5 1e30\nnewmtl Nan\nKd nan 0 0\n");
	struct Case {
		const char *text;
		bool ok;
	} cases[] = {
	    {"mtllib m.mtl\nv 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nusemtl Red\nf 1 2 3\nusemtl Glass\nf 1/1/1 2/2/2 4/4/4 3\n",
	     true},
	    {"mtllib m.mtl\nusemtl Nan\nv 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\r\n", true},
	    {"v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n", false},          // vertex 4 does not exist
	    {"v 0 0 0\nv 1 0 0\nv 0 1 0\nf -1 2 3\n", false},         // negative index
	    {"v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2\n", false},            // two tokens
	    {"v 0 0 0\nv 1 0 0\nv 0 1 0\nf a b c\n", false},          // not numbers
	    {"v 0 0 0\nv 1 0 0\nv 0 1 0\nf 99999999999 1 2\n", false}, // out of int range
	    {"v 0 0\nv 1\nv\nf 1 2 3\n# comment\n\n", true},          // short vertex lines read as 0
	    {"mtllib missing.mtl\nusemtl Whatever\n", false},         // no faces: rejected
	    {"", false},
	};
	for (const Case &c : cases) {
		write(obj, c.text);
		TriangleSet ts;
		std::string err;
		const bool ok = load_obj(obj, 0.35f, ts, err);
		if (ok != c.ok)
			std::printf("loader case returned %d (%s):\n%s\n", ok, err.c_str(), c.text);
		CHECK(ok == c.ok);
		if (ok) {
			CHECK(ts.v.size() == 9 * ts.size() && ts.rgb.size() == 3 * ts.size() && ts.normal.size() == 3 * ts.size());
			tree_case(ts.v);
		} else {
			CHECK(!err.empty());
		}
	}
	TriangleSet ts;
	std::string err;
	CHECK(!load_obj(dir + "/does-not-exist.obj", 1.0f, ts, err));
}

int main(int argc, char **argv) {
	const std::string dir = argc > 1 ? argv[1] : ".";
	loader_cases(dir);
	for (int n : {0, 1, 2, 3, 4, 5, 7, 17, 1000})
		tree_case(soup(n, 11u + static_cast<unsigned>(n), 1.0f));
	tree_case(soup(200, 3u, 1e30f));  // huge coordinates
	tree_case(soup(200, 4u, 1e-30f)); // tiny coordinates
	std::vector<float> same(9 * 50, 0.5f); // every centroid equal, zero-area triangles
	tree_case(same);
	tree_case(soup(300000, 5u, 1.0f)); // large enough for the threaded top levels
	complete_tree_case();
	tile_order_cases();
	std::printf(g_fail ? "FAILED\n" : "host checks passed\n");
	return g_fail;
}
