#include "host_scene.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <thread>

namespace rnb {

namespace {

// glm::min / glm::max on scalars: (y < x) ? y : x and (x < y) ? y : x
// (third_party/glm/detail/func_common.inl:17-30). The comparison order matters
// for signed zeros, so it is kept.
inline float gmin(float x, float y) { return (y < x) ? y : x; }
inline float gmax(float x, float y) { return (x < y) ? y : x; }

// The tree's shape depends only on the triangle count: a range of c > 4 triangles
// splits into c/2 and c - c/2. So every subtree's node count (and depth) is known
// before it is built, each node's pre-order slot can be computed up front, and
// disjoint subtrees can be built on separate threads with the same result.
struct Shape {
	std::map<int, int> nodes, depth;
	int node_count(int c) {
		if (c <= 4)
			return 1;
		auto it = nodes.find(c);
		if (it != nodes.end())
			return it->second;
		const int v = 1 + node_count(c / 2) + node_count(c - c / 2);
		nodes[c] = v;
		return v;
	}
	int depth_of(int c) {
		if (c <= 4)
			return 1;
		auto it = depth.find(c);
		if (it != depth.end())
			return it->second;
		const int v = 1 + std::max(depth_of(c / 2), depth_of(c - c / 2));
		depth[c] = v;
		return v;
	}
};

struct Builder {
	const float *v;
	std::vector<Vec3> centroids;
	Bvh2 *out;
	Shape shape;

	const float *tri(int i) const { return v + 9 * static_cast<size_t>(i); }

	// src/BVH.cpp:18-63, restated: box over the triangles of order[start, start+count),
	// leaf when count <= 4, else nth_element at the median centroid of the widest
	// centroid axis; the node takes pre-order slot `self`, its left subtree the slots
	// after it, its right subtree the slots after those. The top `par_levels` levels
	// build their left subtree on a new thread.
	// Node count of a subtree of c triangles; shape.node_count(n) has filled the
	// table for every size below n before the threads start, so this only reads it.
	int subtree_nodes(int c) const { return c <= 4 ? 1 : shape.nodes.at(c); }

	void build(int self, int start, int count, int par_levels) {
		BvhNode node;
		float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
		for (int i = start; i < start + count; i++) {
			const float *t = tri(out->order[i]);
			for (int k = 0; k < 3; k++)
				for (int a = 0; a < 3; a++) {
					lo[a] = gmin(lo[a], t[3 * k + a]);
					hi[a] = gmax(hi[a], t[3 * k + a]);
				}
		}
		node.bmin = {lo[0], lo[1], lo[2]};
		node.bmax = {hi[0], hi[1], hi[2]};
		if (count <= 4) {
			node.start = start;
			node.count = count;
			out->nodes[static_cast<size_t>(self)] = node;
			return;
		}
		float cmin[3] = {1e30f, 1e30f, 1e30f}, cmax[3] = {-1e30f, -1e30f, -1e30f};
		for (int i = start; i < start + count; i++) {
			const Vec3 &c = centroids[out->order[i]];
			const float cc[3] = {c.x, c.y, c.z};
			for (int a = 0; a < 3; a++) {
				cmin[a] = gmin(cmin[a], cc[a]);
				cmax[a] = gmax(cmax[a], cc[a]);
			}
		}
		const float ex = cmax[0] - cmin[0], ey = cmax[1] - cmin[1], ez = cmax[2] - cmin[2];
		const int axis = (ex > ey && ex > ez) ? 0 : (ey > ez ? 1 : 2);
		const int mid = start + count / 2;
		const Vec3 *cen = centroids.data();
		auto key = [cen, axis](int a) { return axis == 0 ? cen[a].x : (axis == 1 ? cen[a].y : cen[a].z); };
		std::nth_element(out->order.begin() + start, out->order.begin() + mid, out->order.begin() + start + count,
		                 [&key](int a, int b) { return key(a) < key(b); });
		const int nl = mid - start, nr = start + count - mid;
		const int l = self + 1;
		const int r = self + 1 + subtree_nodes(nl);
		node.count = 0;
		node.left = l;
		node.right = r;
		out->nodes[static_cast<size_t>(self)] = node;
		if (par_levels > 0) {
			std::thread left([this, l, start, nl, par_levels] { build(l, start, nl, par_levels - 1); });
			build(r, mid, nr, par_levels - 1);
			left.join();
		} else {
			build(l, start, nl, 0);
			build(r, mid, nr, 0);
		}
	}
};

} // namespace

void build_reference_bvh(const float *v9, int n, Bvh2 &out) {
	out.order.resize(static_cast<size_t>(n));
	out.nodes.clear();
	out.root = -1;
	out.depth = 0;
	Builder b;
	b.v = v9;
	b.out = &out;
	b.centroids.resize(static_cast<size_t>(n));
	// centroid = (v0 + v1 + v2) / 3.0f, component-wise in that order (src/BVH.cpp:10-13).
	for (int i = 0; i < n; i++) {
		out.order[i] = i;
		const float *t = v9 + 9 * static_cast<size_t>(i);
		b.centroids[i] = {((t[0] + t[3]) + t[6]) / 3.0f, ((t[1] + t[4]) + t[7]) / 3.0f, ((t[2] + t[5]) + t[8]) / 3.0f};
	}
	if (n > 0) {
		out.nodes.resize(static_cast<size_t>(b.shape.node_count(n)));
		out.depth = b.shape.depth_of(n);
		// Threads only where subtrees are large enough to repay them.
		const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
		int par = 0;
		while ((1u << par) < 2 * hw && (n >> par) > 65536)
			par++;
		b.build(0, 0, n, par);
		out.root = 0;
	}
}

Vec3 loader_face_normal(const float *t) {
	// cross(v1 - v0, v2 - v0), divided by its length when > 1e-8, else (0,1,0).
	const float ax = t[3] - t[0], ay = t[4] - t[1], az = t[5] - t[2];
	const float bx = t[6] - t[0], by = t[7] - t[1], bz = t[8] - t[2];
	const float cx = ay * bz - by * az, cy = az * bx - bz * ax, cz = ax * by - bx * ay;
	const float len = std::sqrt((cx * cx + cy * cy) + cz * cz);
	if (len > 1e-8f)
		return {cx / len, cy / len, cz / len};
	return {0.0f, 1.0f, 0.0f};
}

static void cross_d(const float *t, double c[3]) {
	const double ax = static_cast<double>(t[3]) - t[0], ay = static_cast<double>(t[4]) - t[1],
	             az = static_cast<double>(t[5]) - t[2];
	const double bx = static_cast<double>(t[6]) - t[0], by = static_cast<double>(t[7]) - t[1],
	             bz = static_cast<double>(t[8]) - t[2];
	c[0] = ay * bz - az * by;
	c[1] = az * bx - ax * bz;
	c[2] = ax * by - ay * bx;
}

Vec3 geometric_normal(const float *t) {
	double c[3];
	cross_d(t, c);
	const double len = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
	if (!(len > 0.0))
		return {0.0f, 0.0f, 0.0f};
	return {static_cast<float>(c[0] / len), static_cast<float>(c[1] / len), static_cast<float>(c[2] / len)};
}

double triangle_area(const float *t) {
	double c[3];
	cross_d(t, c);
	return 0.5 * std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
}

namespace {

int materialFor(const std::string &name) {
	if (name == "Mirror")
		return kRefMirror;
	if (name == "Glass")
		return kRefGlass;
	if (name == "Marble")
		return kRefProcedural;
	if (name == "Bumpy")
		return kRefBump;
	if (name == "Parallax")
		return kRefParallax;
	if (name == "Metal")
		return kRefMetal;
	if (name == "Dispersive" || name == "Prism")
		return kRefDispersive;
	if (name == "Subsurface" || name == "SSS" || name == "Wax" || name == "Jade")
		return kRefSubsurface;
	if (name == "NormalMap" || name == "Normal")
		return kRefNormalMap;
	if (name == "Emissive" || name == "Emit" || name == "Glow")
		return kRefEmissive;
	return kRefDiffuse;
}

struct Mtl {
	int r = 0, g = 0, b = 0;
};

// int(x) as the reference's x86-64 build converts (cvttss2si): truncation, and
// INT_MIN for NaN and values outside the int range (a C++ cast would be undefined).
int x86_float_to_int(float x) {
	return (x >= -2147483648.0f && x < 2147483648.0f) ? static_cast<int>(x) : static_cast<int>(0x80000000u);
}

bool parse_int_prefix(const std::string &s, int &out) {
	// std::stoi semantics on the leading integer (leading spaces and sign allowed).
	const char *p = s.c_str();
	char *end = nullptr;
	errno = 0;
	long v = std::strtol(p, &end, 10);
	if (end == p || errno != 0 || v < -2147483647L || v > 2147483647L)
		return false;
	out = static_cast<int>(v);
	return true;
}

bool parse_face_vertex(const std::string &tok, int &v) {
	size_t slash = tok.find('/');
	return parse_int_prefix(slash == std::string::npos ? tok : tok.substr(0, slash), v) && (v -= 1, true);
}

std::map<std::string, Mtl> load_mtl(const std::string &path) {
	std::map<std::string, Mtl> out;
	std::ifstream f(path);
	if (!f.is_open())
		return out;
	std::string line, cur;
	while (std::getline(f, line)) {
		std::stringstream ss(line);
		std::string type;
		ss >> type;
		if (type == "newmtl") {
			ss >> cur;
		} else if (type == "Kd" && !cur.empty()) {
			float r = 0, g = 0, b = 0;
			ss >> r >> g >> b;
			Mtl m;
			m.r = x86_float_to_int(r * 255);
			m.g = x86_float_to_int(g * 255);
			m.b = x86_float_to_int(b * 255);
			out[cur] = m;
		}
	}
	return out;
}

} // namespace

bool load_obj(const std::string &path, float scale, TriangleSet &ts, std::string &err) {
	std::ifstream f(path);
	if (!f.is_open()) {
		err = "cannot open " + path;
		return false;
	}
	std::string dir;
	size_t slash = path.find_last_of("/\\");
	if (slash != std::string::npos)
		dir = path.substr(0, slash + 1);
	std::map<std::string, Mtl> mtls;
	std::vector<float> verts;
	struct Face {
		int a, b, c, r, g, bl, mat;
	};
	std::vector<Face> faces;
	int cr = 0, cg = 0, cb = 0, cmat = kRefDiffuse;
	std::string line;
	while (std::getline(f, line)) {
		std::stringstream ss(line);
		std::string type;
		ss >> type;
		if (type == "mtllib") {
			std::string name;
			ss >> name;
			mtls = load_mtl(dir + name);
		} else if (type == "usemtl") {
			std::string name;
			ss >> name;
			cmat = materialFor(name);
			auto it = mtls.find(name);
			if (it != mtls.end()) {
				cr = it->second.r;
				cg = it->second.g;
				cb = it->second.b;
			}
		} else if (type == "v") {
			float x = 0, y = 0, z = 0;
			ss >> x >> y >> z;
			verts.push_back(x * scale);
			verts.push_back(y * scale);
			verts.push_back(z * scale);
		} else if (type == "f") {
			std::string t1, t2, t3;
			ss >> t1 >> t2 >> t3;
			Face fc{};
			if (!parse_face_vertex(t1, fc.a) || !parse_face_vertex(t2, fc.b) || !parse_face_vertex(t3, fc.c)) {
				err = "malformed face line: " + line;
				return false;
			}
			fc.r = cr;
			fc.g = cg;
			fc.bl = cb;
			fc.mat = cmat;
			faces.push_back(fc);
		}
	}
	const long nv = static_cast<long>(verts.size() / 3);
	ts = TriangleSet();
	ts.v.reserve(faces.size() * 9);
	for (const Face &fc : faces) {
		for (int idx : {fc.a, fc.b, fc.c}) {
			if (idx < 0 || idx >= nv) {
				err = "face references a vertex that does not exist";
				return false;
			}
			ts.v.push_back(verts[3 * idx]);
			ts.v.push_back(verts[3 * idx + 1]);
			ts.v.push_back(verts[3 * idx + 2]);
		}
		ts.rgb.push_back(fc.r);
		ts.rgb.push_back(fc.g);
		ts.rgb.push_back(fc.bl);
		ts.ref_material.push_back(fc.mat);
		ts.roughness.push_back(0.2f);
	}
	const size_t n = faces.size();
	ts.normal.resize(3 * n);
	for (size_t i = 0; i < n; i++) {
		Vec3 nn = loader_face_normal(&ts.v[9 * i]);
		ts.normal[3 * i] = nn.x;
		ts.normal[3 * i + 1] = nn.y;
		ts.normal[3 * i + 2] = nn.z;
	}
	if (n == 0) {
		err = "no faces in " + path;
		return false;
	}
	// Vertex normals (src/ObjLoader.cpp:178-204): per face corner, the normalised sum
	// of the normals of the faces sharing that OBJ vertex whose normal is within
	// about 60 degrees (dot > 0.5) of this face's, in face order; the face normal
	// when the sum vanishes.
	std::vector<std::vector<int>> vertex_faces(static_cast<size_t>(nv));
	for (size_t i = 0; i < n; i++)
		for (int idx : {faces[i].a, faces[i].b, faces[i].c})
			vertex_faces[static_cast<size_t>(idx)].push_back(static_cast<int>(i));
	auto fn = [&ts](int i) -> Vec3 {
		return {ts.normal[3 * static_cast<size_t>(i)], ts.normal[3 * static_cast<size_t>(i) + 1],
		        ts.normal[3 * static_cast<size_t>(i) + 2]};
	};
	auto dot3 = [](Vec3 a, Vec3 b) {
		const float x = a.x * b.x, y = a.y * b.y, z = a.z * b.z;
		return (x + y) + z;
	};
	ts.vnormal.resize(9 * n);
	for (size_t i = 0; i < n; i++) {
		const Vec3 own = fn(static_cast<int>(i));
		const int corner[3] = {faces[i].a, faces[i].b, faces[i].c};
		for (int k = 0; k < 3; k++) {
			Vec3 sum{0.0f, 0.0f, 0.0f};
			for (int g : vertex_faces[static_cast<size_t>(corner[k])]) {
				const Vec3 o = fn(g);
				if (dot3(o, own) > 0.5f)
					sum = {sum.x + o.x, sum.y + o.y, sum.z + o.z};
			}
			Vec3 out = own;
			if (std::sqrt(dot3(sum, sum)) > 0.0f) {
				const float inv = 1.0f / std::sqrt(dot3(sum, sum));
				out = {sum.x * inv, sum.y * inv, sum.z * inv};
			}
			ts.vnormal[9 * i + 3 * k] = out.x;
			ts.vnormal[9 * i + 3 * k + 1] = out.y;
			ts.vnormal[9 * i + 3 * k + 2] = out.z;
		}
	}
	return true;
}

void flatten_bvh4(const Bvh2 &bvh, DeviceLayout4 &out) {
	out.nodes.clear();
	if (bvh.root < 0)
		return;
	auto as_float = [](int i) {
		float f;
		std::memcpy(&f, &i, 4);
		return f;
	};
	auto leaf_ref = [&](const BvhNode &nd) { return ~((nd.start << 3) | nd.count); };
	const BvhNode &root = bvh.nodes[static_cast<size_t>(bvh.root)];
	if (root.count > 0) {
		out.root_ref = leaf_ref(root);
		return;
	}
	// Which reference levels become 4-wide nodes. Every node spans two reference
	// levels at most, and any such frontier gives the same traversal result, so the
	// choice only moves cost: each 4-wide node costs one fetch per ray that reaches
	// it, about in proportion to its box's surface area. Bottom-up over the tree,
	// F(n) = area(n) + sum over n's children c of G(c) is the cost below n when n
	// roots a 4-wide node, and G(c) = min(F(c), F of c's internal children) picks,
	// per internal child, between keeping it as an entry and splicing its two
	// children in. On a complete tree of odd height this puts the 4-wide nodes at
	// even heights above the leaves (all nodes full, about half as many) where a
	// top-down collapse leaves the bottom level half empty.
	const size_t nn = bvh.nodes.size();
	std::vector<double> cost_root(nn, 0.0), cost_best(nn, 0.0);
	std::vector<char> splice(nn, 0);
	{
		auto area = [](const BvhNode &nd) {
			const double x = std::max(0.0, static_cast<double>(nd.bmax.x) - nd.bmin.x);
			const double y = std::max(0.0, static_cast<double>(nd.bmax.y) - nd.bmin.y);
			const double z = std::max(0.0, static_cast<double>(nd.bmax.z) - nd.bmin.z);
			return x * y + y * z + z * x;
		};
		std::vector<int> pre; // pre-order; walked backwards, children come before parents
		std::vector<int> st{bvh.root};
		while (!st.empty()) {
			const int i = st.back();
			st.pop_back();
			pre.push_back(i);
			const BvhNode &nd = bvh.nodes[static_cast<size_t>(i)];
			if (nd.count == 0) {
				st.push_back(nd.left);
				st.push_back(nd.right);
			}
		}
		auto internal_root_cost = [&](int c) {
			return bvh.nodes[static_cast<size_t>(c)].count > 0 ? 0.0 : cost_root[static_cast<size_t>(c)];
		};
		for (size_t k = pre.size(); k-- > 0;) {
			const int i = pre[k];
			const BvhNode &nd = bvh.nodes[static_cast<size_t>(i)];
			if (nd.count > 0)
				continue;
			const size_t l = static_cast<size_t>(nd.left), r = static_cast<size_t>(nd.right);
			const bool leaf_l = bvh.nodes[l].count > 0, leaf_r = bvh.nodes[r].count > 0;
			cost_root[static_cast<size_t>(i)] =
			    area(nd) + (leaf_l ? 0.0 : cost_best[l]) + (leaf_r ? 0.0 : cost_best[r]);
			const double spliced = internal_root_cost(nd.left) + internal_root_cost(nd.right);
			splice[static_cast<size_t>(i)] = spliced < cost_root[static_cast<size_t>(i)];
			cost_best[static_cast<size_t>(i)] = std::min(cost_root[static_cast<size_t>(i)], spliced);
		}
	}
	// Iterative build: each work item fills node `slot` from reference node `src`.
	std::vector<std::pair<int, int>> work; // (slot, src)
	out.nodes.resize(8);
	work.push_back({0, bvh.root});
	while (!work.empty()) {
		const auto [slot, src] = work.back();
		work.pop_back();
		const BvhNode &n = bvh.nodes[static_cast<size_t>(src)];
		// Entries in pop order: right side first, and within a side its right child first.
		int ent[4];
		int cnt = 0;
		for (int c : {n.right, n.left}) {
			const BvhNode &cn = bvh.nodes[static_cast<size_t>(c)];
			if (cn.count > 0 || !splice[static_cast<size_t>(c)]) {
				ent[cnt++] = c;
			} else {
				ent[cnt++] = cn.right;
				ent[cnt++] = cn.left;
			}
		}
		float lo[3][4], hi[3][4];
		int refs[4];
		for (int k = 0; k < 4; k++) {
			for (int a = 0; a < 3; a++) {
				lo[a][k] = 1.0f;
				hi[a][k] = -1.0f;
			}
			refs[k] = 0;
		}
		for (int k = 0; k < cnt; k++) {
			const BvhNode &e = bvh.nodes[static_cast<size_t>(ent[k])];
			lo[0][k] = e.bmin.x;
			lo[1][k] = e.bmin.y;
			lo[2][k] = e.bmin.z;
			hi[0][k] = e.bmax.x;
			hi[1][k] = e.bmax.y;
			hi[2][k] = e.bmax.z;
			if (e.count > 0) {
				refs[k] = leaf_ref(e);
			} else {
				const int child_slot = static_cast<int>(out.nodes.size() / 8);
				out.nodes.resize(out.nodes.size() + 8);
				refs[k] = child_slot;
				work.push_back({child_slot, ent[k]});
			}
		}
		F4 *o = &out.nodes[static_cast<size_t>(slot) * 8];
		// (lo, hi) pairs per axis and entry, two entries per float4.
		for (int a = 0; a < 3; a++) {
			o[2 * a] = {lo[a][0], hi[a][0], lo[a][1], hi[a][1]};
			o[2 * a + 1] = {lo[a][2], hi[a][2], lo[a][3], hi[a][3]};
		}
		o[6] = {as_float(refs[0]), as_float(refs[1]), as_float(refs[2]), as_float(refs[3])};
		o[7] = {as_float(cnt), 0.0f, 0.0f, 0.0f};
	}
	out.root_ref = 0;
}

void flatten_bvh(const TriangleSet &ts, const Bvh2 &bvh, DeviceLayout &out) {
	const int n = static_cast<int>(ts.size());
	out.nodes.clear();
	out.tris.assign(static_cast<size_t>(n) * 3, F4{0, 0, 0, 0});
	out.depth = bvh.depth;
	// Dense indices for internal nodes, in reference node order.
	std::vector<int> dense(bvh.nodes.size(), -1);
	int ni = 0;
	for (size_t i = 0; i < bvh.nodes.size(); i++)
		if (bvh.nodes[i].count == 0)
			dense[i] = ni++;
	out.internal_count = ni;
	auto ref_of = [&](int node) -> int {
		const BvhNode &nd = bvh.nodes[static_cast<size_t>(node)];
		if (nd.count > 0)
			return ~((nd.start << 3) | nd.count);
		return dense[static_cast<size_t>(node)];
	};
	auto as_float = [](int i) {
		float f;
		std::memcpy(&f, &i, 4);
		return f;
	};
	out.nodes.resize(static_cast<size_t>(ni) * 4);
	for (size_t i = 0; i < bvh.nodes.size(); i++) {
		const BvhNode &nd = bvh.nodes[i];
		if (nd.count > 0)
			continue;
		const BvhNode &L = bvh.nodes[static_cast<size_t>(nd.left)];
		const BvhNode &R = bvh.nodes[static_cast<size_t>(nd.right)];
		F4 *o = &out.nodes[static_cast<size_t>(dense[i]) * 4];
		o[0] = {L.bmin.x, L.bmax.x, L.bmin.y, L.bmax.y};
		o[1] = {R.bmin.x, R.bmax.x, R.bmin.y, R.bmax.y};
		o[2] = {L.bmin.z, L.bmax.z, R.bmin.z, R.bmax.z};
		o[3] = {as_float(ref_of(nd.left)), as_float(ref_of(nd.right)), 0.0f, 0.0f};
	}
	if (bvh.root >= 0) {
		const BvhNode &r = bvh.nodes[static_cast<size_t>(bvh.root)];
		out.root_lo[0] = r.bmin.x;
		out.root_lo[1] = r.bmin.y;
		out.root_lo[2] = r.bmin.z;
		out.root_hi[0] = r.bmax.x;
		out.root_hi[1] = r.bmax.y;
		out.root_hi[2] = r.bmax.z;
		out.root_ref = ref_of(bvh.root);
	} else {
		for (int a = 0; a < 3; a++) {
			out.root_lo[a] = 1.0f;
			out.root_hi[a] = -1.0f;
		}
		out.root_ref = 0;
	}
	// Static traversal rank: the reference pushes left then right and pops the
	// right child first, so leaves are met in that order (src/BVH.cpp:77-111).
	std::vector<int> rank_of_pos(static_cast<size_t>(n), 0);
	if (bvh.root >= 0) {
		std::vector<int> st;
		st.push_back(bvh.root);
		int next = 0;
		while (!st.empty()) {
			int k = st.back();
			st.pop_back();
			const BvhNode &nd = bvh.nodes[static_cast<size_t>(k)];
			if (nd.count > 0) {
				for (int p = nd.start; p < nd.start + nd.count; p++)
					rank_of_pos[static_cast<size_t>(p)] = next++;
			} else {
				st.push_back(nd.left);
				st.push_back(nd.right);
			}
		}
	}
	for (int p = 0; p < n; p++) {
		const int ti = bvh.order[static_cast<size_t>(p)];
		const float *t = &ts.v[9 * static_cast<size_t>(ti)];
		F4 *o = &out.tris[3 * static_cast<size_t>(p)];
		o[0] = {t[0], t[1], t[2], as_float(ti)};
		o[1] = {t[3] - t[0], t[4] - t[1], t[5] - t[2], as_float(rank_of_pos[static_cast<size_t>(p)])};
		o[2] = {t[6] - t[0], t[7] - t[1], t[8] - t[2], 0.0f};
	}
}

} // namespace rnb
