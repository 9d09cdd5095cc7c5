// Host-side scene representation, reference-identical BVH build and the
// flattening of that BVH into the device layout read by the CUDA kernels.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace rnb {

// Surface responses of the reference renderer, same order as its Material enum
// (framework/ModelTriangle.h:12-24).
enum RefMaterial : int {
	kRefDiffuse = 0,
	kRefMirror = 1,
	kRefGlass = 2,
	kRefProcedural = 3,
	kRefBump = 4,
	kRefParallax = 5,
	kRefMetal = 6,
	kRefDispersive = 7,
	kRefSubsurface = 8,
	kRefNormalMap = 9,
	kRefEmissive = 10,
};

// Physical-mode BSDFs (the additive path-tracing API).
enum PhysMaterial : int { kLambert = 0, kGGX = 1, kDielectric = 2 };

struct Vec3 {
	float x, y, z;
};

// Triangle list in structure-of-arrays form. `v` holds 9 floats per triangle.
// The reference fields (rgb/material/roughness/normal) drive the drop-in
// reference-mode renderer; the physical fields drive the additive API.
struct TriangleSet {
	std::vector<float> v;           // 9 per triangle: v0, v1, v2
	std::vector<int> rgb;           // 3 per triangle, reference Colour 0..255
	std::vector<int> ref_material;  // reference Material code
	std::vector<float> roughness;   // reference Metal roughness (default 0.2)
	std::vector<float> normal;      // 3 per triangle, face normal as the loader computes it
	std::vector<float> vnormal;     // 9 per triangle, vertex normals (ModelTriangle::vertexNormals)
	std::vector<float> albedo;      // 3 per triangle (physical mode)
	std::vector<float> emission;    // 3 per triangle (physical mode, Le)
	std::vector<int> phys_material; // PhysMaterial
	std::vector<float> phys_param;  // GGX alpha or dielectric IOR
	size_t size() const { return v.size() / 9; }
};

// Reference BVH node (src/BVH.h:22-26): box, children or a leaf range in `order`.
struct BvhNode {
	Vec3 bmin, bmax;
	int left = -1, right = -1;
	int start = 0, count = 0;
};

struct Bvh2 {
	std::vector<int> order;
	std::vector<BvhNode> nodes;
	int root = -1;
	int depth = 0; // maximum root-to-leaf depth (root = 1)
};

// Median-split build with leaves of <= 4 triangles, identical node order and
// triangle order to the reference (src/BVH.cpp:6-63).
void build_reference_bvh(const float *v9, int n, Bvh2 &out);

// Face normal as the reference OBJ loader computes it (src/ObjLoader.cpp:170-176).
Vec3 loader_face_normal(const float *v9);

// Unit geometric normal cross(v1 - v0, v2 - v0) (computed in double, rounded
// once), (0, 0, 0) for a degenerate triangle; and the triangle's area.
Vec3 geometric_normal(const float *v9);
double triangle_area(const float *v9);

// Wavefront OBJ/MTL loader with the reference loader's semantics
// (src/ObjLoader.cpp:23-214): `v` scaled by `scale`, first three face tokens,
// `usemtl` name -> Material mapping and Kd colour as int(Kd*255).
bool load_obj(const std::string &path, float scale, TriangleSet &out, std::string &err);

// Device layout of a flattened reference BVH.
//  nodes: 4 float4 per internal node ("child pair" node):
//     n0 = (L.lo.x, L.hi.x, L.lo.y, L.hi.y)
//     n1 = (R.lo.x, R.hi.x, R.lo.y, R.hi.y)
//     n2 = (L.lo.z, L.hi.z, R.lo.z, R.hi.z)
//     n3 = (ref L, ref R, -, -) as int bits
//  child ref >= 0: dense internal node index; ref < 0: leaf ~((start << 3) | count)
//  tris: 3 float4 per triangle position in leaf order:
//     (v0.xyz, original index), (e0 = v1 - v0, rank), (e1 = v2 - v0, 0)
//  rank = position of the triangle in the reference's static traversal order
//  (leaves visited right child first, triangles ascending within a leaf).
struct F4 {
	float x, y, z, w;
};
struct DeviceLayout {
	std::vector<F4> nodes;
	std::vector<F4> tris;
	float root_lo[3], root_hi[3];
	int root_ref = 0;
	int internal_count = 0;
	int depth = 0;
};
void flatten_bvh(const TriangleSet &ts, const Bvh2 &bvh, DeviceLayout &out);

// Four-wide collapse of the same tree for the fast traversal. A node holds the
// children of one reference node, with an internal child either kept as an entry
// or replaced by its own two children (so two to four entries), in the order the
// reference pops them; which children are replaced is chosen bottom-up by an
// area-weighted fetch cost. refs are int bits (>= 0 node, < 0 leaf as in the
// 2-wide layout).
// Boxes are the reference's own node boxes. Because float subtraction and
// multiplication round monotonically, a grandchild's slab interval lies inside
// its parent's, so skipping the parent's test never admits a node the
// reference would prune (rays with an infinite 1/d component excepted: those
// use the 2-wide layout).
// Node rows: [2a] = (lo_a[0], hi_a[0], lo_a[1], hi_a[1]), [2a+1] = entries 2, 3,
// for axis a = x, y, z; [6] = refs[4]; [7] = (count, 0, 0, 0).
struct DeviceLayout4 {
	std::vector<F4> nodes;
	int root_ref = 0; // node index, or a leaf ref when the reference root is a leaf
};
void flatten_bvh4(const Bvh2 &bvh, DeviceLayout4 &out);

} // namespace rnb
