// Device-resident scene layout, shared by the host flattener and the CUDA kernels.
//
// Everything a ray touches in its inner loop is 16-byte aligned and read with
// 128-bit loads:
//   DevNode      64 B  both children's boxes of one interior node of the
//                      reference's binary SAH BVH (same topology, child-box form)
//   DevTriangle  48 B  three vertices of one triangle, in BVH leaf order
//   DevObject    16 B  one TLAS primitive (sphere, triangle or instance), leaf order
//   DevSphere    16 B  center and radius
//   DevInstance 112 B  object-to-world and world-to-object 3x4 rows, BLAS root
// Shading-only data (texture coordinates, corner normals, materials, lights) sits
// in separate tables read once per hit.
#pragma once

#include <cstdint>

namespace albedo_b200 {

// A child reference in a DevNode.
//   bit 31 clear: an interior node index.
//   bit 31 set:   a leaf: bits 0..27 first primitive (leaf-order index),
//                 bits 28..30 primitive count - 1 (leaves hold 1..4).
// kEmptyChild (count field 7) marks a missing child (a root that is a leaf).
constexpr std::uint32_t kLeafBit{0x80000000u};
constexpr std::uint32_t kLeafFirstMask{0x0FFFFFFFu};
constexpr std::uint32_t kEmptyChild{0xFFFFFFFFu};
constexpr std::uint32_t kMaxLeafFirst{kLeafFirstMask};

// A 4-wide node: two levels of the reference's binary BVH collapsed into one.
// Child i's box is (lo_x[i], hi_x[i], lo_y[i], ...); absent children are
// kEmptyChild. `order[o]` lists, for the ray octant o (bit a set when the
// direction's component a is negative), the children in the order the
// reference's depth-first, near-first traversal reaches them: 2 bits per child,
// nearest first, low bits first.
struct alignas(16) DevNode {
    float lo_x[4];
    float hi_x[4];
    float lo_y[4];
    float hi_y[4];
    float lo_z[4];
    float hi_z[4];
    std::uint32_t child[4];
    std::uint8_t order[8];
    std::uint32_t count;  // children present (1..4); they are child[0..count-1]
    std::uint32_t groups; // slots per binary child of the collapsed node (bits 0-1, 2-3); 0 for a leaf root
};
static_assert(sizeof(DevNode) == 128);

// v0.w holds the triangle's index within its mesh (or, for scene triangles, its
// index in the scene triangle table) as raw bits.
struct alignas(16) DevTriangle {
    float v0x, v0y, v0z, v0w;
    float v1x, v1y, v1z, v1w;
    float v2x, v2y, v2z, v2w;
};
static_assert(sizeof(DevTriangle) == 48);

// Per-triangle shading attributes, in the same leaf order as DevTriangle:
// front normal, smooth flag, corner texture coordinates and corner normals.
struct alignas(16) DevTriangleAttr {
    float nx, ny, nz, smooth;
    float u0, v0, u1, v1;
    float u2, v2, cn0x, cn0y;
    float cn0z, cn1x, cn1y, cn1z;
    float cn2x, cn2y, cn2z, pad;
};
static_assert(sizeof(DevTriangleAttr) == 80);

enum DevObjectKind : std::uint32_t {
    kObjSphere = 0,      // FP32 quadratic
    kObjTriangle = 1,
    kObjInstance = 2,
    kObjSphereWide = 3,  // sphere whose coordinates need the FP64 quadratic
};

struct alignas(16) DevObject {
    std::uint32_t kind;     // DevObjectKind
    std::uint32_t index;    // sphere, scene-triangle (leaf position) or instance index
    std::uint32_t material;
    std::uint32_t id;       // object id in add order (HitRecord::object)
};

struct alignas(16) DevSphere {
    float cx, cy, cz, r;
};

struct alignas(16) DevInstance {
    float to_object[12]; // rows: l00 l01 l02 o0 | l10 l11 l12 o1 | l20 l21 l22 o2
    float to_world[12];
    std::uint32_t root;   // BLAS root node index in the node table
    std::uint32_t mesh;
    std::uint32_t pad0, pad1;
};
static_assert(sizeof(DevInstance) == 112);

enum DevTexture : std::uint32_t { kTexConstant = 0, kTexChecker = 1, kTexPerlin = 2 };
enum DevBasicKind : std::uint32_t { kDiffuse = 0, kConductor = 1, kDielectric = 2 };

// One basic material.
//   diffuse:    texture, a = color / even / low, b = odd / high, s0 = frequency / scale, s1 = veins
//   conductor:  a = eta, b = k, s0 = alpha (roughness squared)
//   dielectric: s0 = alpha, s1 = ior
struct alignas(16) DevBasic {
    std::uint32_t kind;
    std::uint32_t texture;
    float s0, s1;
    float a[3];
    float pad0;
    float b[3];
    float pad1;
};
static_assert(sizeof(DevBasic) == 48);

struct alignas(16) DevMaterial {
    std::uint32_t mix; // 0: `first` only; 1: Perlin mix of first and second
    float scale, veins, threshold;
    DevBasic first;
    DevBasic second;
};
static_assert(sizeof(DevMaterial) == 112);

enum DevLightKind : std::uint32_t { kLightPoint = 0, kLightArea = 1, kLightSky = 2 };

//   point: p = position, e = intensity
//   area:  p = center, radius, e = radiance, object = its surface's object id
//   sky:   e = nadir, z = zenith
struct alignas(16) DevLight {
    std::uint32_t kind;
    std::uint32_t object;
    float radius, pad0;
    float p[3];
    float pad1;
    float e[3];
    float pad2;
    float z[3];
    float pad3;
};
static_assert(sizeof(DevLight) == 64);

struct DevCamera {
    float origin[3];
    float forward[3];
    float half_width[3];
    float half_height[3];
};

// Device pointers and counts of one uploaded scene.
struct DevScene {
    const DevNode* nodes;
    const DevObject* objects;          // TLAS leaf order
    const DevSphere* spheres;
    const DevTriangle* triangles;      // scene triangles then every mesh's triangles, leaf order
    const DevTriangleAttr* attrs;      // parallel to triangles
    const DevInstance* instances;
    const DevMaterial* materials;
    const DevLight* lights;
    const std::int32_t* object_light;  // object id -> area light index or -1
    const double* instance_to_object64; // per instance, the exact FP64 world-to-object 3x4 rows (hit refinement)
    std::uint32_t tlas_root;           // node index of the TLAS root (kEmptyChild if no objects)
    std::uint32_t light_count;
    std::int32_t sky_light;            // light index of the sky, or -1
    std::uint32_t object_count;
};

} // namespace albedo_b200
