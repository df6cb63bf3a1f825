// Flattening: the reference-topology BVHs become child-box nodes over FP32 boxes
// rounded outward; primitives are stored in leaf order so a leaf is one
// contiguous run; everything else becomes flat FP32 tables.
#include "flatten.hpp"

#include <bit>
#include <cmath>
#include <format>
#include <stdexcept>

namespace albedo_b200 {

namespace {

// The largest float <= x and the smallest float >= x.
float roundDown(double x)
{
    float f{static_cast<float>(x)};
    if (static_cast<double>(f) > x) {
        f = std::nextafter(f, -INFINITY);
    }
    return f;
}
float roundUp(double x)
{
    float f{static_cast<float>(x)};
    if (static_cast<double>(f) < x) {
        f = std::nextafter(f, INFINITY);
    }
    return f;
}

std::uint32_t leafRef(std::uint64_t first, std::uint32_t count)
{
    if (first > kMaxLeafFirst) {
        throw std::invalid_argument{std::format("scene has more than {} primitives", kMaxLeafFirst)};
    }
    return kLeafBit | ((count - 1u) << 28) | static_cast<std::uint32_t>(first);
}

void setChildBox(DevNode& node, int child, const Box3& box)
{
    if (child == 0) {
        node.c0_lo_x = roundDown(box.min.x);
        node.c0_hi_x = roundUp(box.max.x);
        node.c0_lo_y = roundDown(box.min.y);
        node.c0_hi_y = roundUp(box.max.y);
        node.c0_lo_z = roundDown(box.min.z);
        node.c0_hi_z = roundUp(box.max.z);
    } else {
        node.c1_lo_x = roundDown(box.min.x);
        node.c1_hi_x = roundUp(box.max.x);
        node.c1_lo_y = roundDown(box.min.y);
        node.c1_hi_y = roundUp(box.max.y);
        node.c1_lo_z = roundDown(box.min.z);
        node.c1_hi_z = roundUp(box.max.z);
    }
}

// Emits the interior nodes of `bvh` (depth-first, first child at i + 1) as
// child-box nodes; leaves index primitives from `prim_base` in leaf order.
// Returns the device index of the root. A root that is itself a leaf gets a
// node whose second child is empty.
std::uint32_t emitBvh(const BuiltBvh& bvh, std::uint64_t prim_base, std::vector<DevNode>& out)
{
    const std::size_t n{bvh.nodes.size()};
    std::vector<std::uint32_t> device_index(n, kEmptyChild);
    const auto base{static_cast<std::uint32_t>(out.size())};
    std::uint32_t next{base};
    for (std::size_t i{0}; i < n; ++i) {
        if (bvh.nodes[i].count == 0) {
            device_index[i] = next++;
        }
    }
    const auto childRef = [&](std::size_t i) {
        const BuildNode& node{bvh.nodes[i]};
        return node.count != 0 ? leafRef(prim_base + node.offset, node.count) : device_index[i];
    };
    if (n == 0) {
        return kEmptyChild;
    }
    if (bvh.nodes[0].count != 0) {
        DevNode root{};
        setChildBox(root, 0, bvh.nodes[0].bounds);
        setChildBox(root, 1, Box3{{0, 0, 0}, {0, 0, 0}});
        root.child0 = childRef(0);
        root.child1 = kEmptyChild;
        root.axis = 0;
        out.push_back(root);
        return base;
    }
    out.resize(next);
    for (std::size_t i{0}; i < n; ++i) {
        const BuildNode& node{bvh.nodes[i]};
        if (node.count != 0) {
            continue;
        }
        DevNode& dev{out[device_index[i]]};
        const std::size_t first{i + 1};
        const std::size_t second{static_cast<std::size_t>(node.offset)};
        setChildBox(dev, 0, bvh.nodes[first].bounds);
        setChildBox(dev, 1, bvh.nodes[second].bounds);
        dev.child0 = childRef(first);
        dev.child1 = childRef(second);
        dev.axis = node.axis;
        dev.pad = 0;
    }
    return base;
}

float f32(double x) { return static_cast<float>(x); }

void putRgb(float* out, const Rgb& c)
{
    out[0] = f32(c.r);
    out[1] = f32(c.g);
    out[2] = f32(c.b);
}

DevTriangle deviceTriangle(const TriangleDesc& t, std::uint32_t id)
{
    DevTriangle d{};
    d.v0x = f32(t.v[0].x);
    d.v0y = f32(t.v[0].y);
    d.v0z = f32(t.v[0].z);
    d.v0w = std::bit_cast<float>(id);
    d.v1x = f32(t.v[1].x);
    d.v1y = f32(t.v[1].y);
    d.v1z = f32(t.v[1].z);
    d.v2x = f32(t.v[2].x);
    d.v2y = f32(t.v[2].y);
    d.v2z = f32(t.v[2].z);
    return d;
}

DevTriangleAttr deviceAttr(const TriangleDesc& t, const std::array<Vec3, 3>* corners)
{
    DevTriangleAttr a{};
    a.nx = f32(t.normal.x);
    a.ny = f32(t.normal.y);
    a.nz = f32(t.normal.z);
    a.smooth = corners != nullptr ? 1.0f : 0.0f;
    a.u0 = f32(t.uv[0][0]);
    a.v0 = f32(t.uv[0][1]);
    a.u1 = f32(t.uv[1][0]);
    a.v1 = f32(t.uv[1][1]);
    a.u2 = f32(t.uv[2][0]);
    a.v2 = f32(t.uv[2][1]);
    if (corners != nullptr) {
        a.cn0x = f32((*corners)[0].x);
        a.cn0y = f32((*corners)[0].y);
        a.cn0z = f32((*corners)[0].z);
        a.cn1x = f32((*corners)[1].x);
        a.cn1y = f32((*corners)[1].y);
        a.cn1z = f32((*corners)[1].z);
        a.cn2x = f32((*corners)[2].x);
        a.cn2y = f32((*corners)[2].y);
        a.cn2z = f32((*corners)[2].z);
    }
    return a;
}

DevBasic deviceBasic(const BasicMaterialDesc& b)
{
    DevBasic d{};
    d.kind = static_cast<std::uint32_t>(b.kind);
    d.texture = static_cast<std::uint32_t>(b.texture.kind);
    switch (b.kind) {
    case BasicKind::Diffuse:
        putRgb(d.a, b.texture.a);
        putRgb(d.b, b.texture.b);
        d.s0 = f32(b.texture.frequency_or_scale);
        d.s1 = f32(b.texture.veins);
        break;
    case BasicKind::Conductor:
        putRgb(d.a, b.eta);
        putRgb(d.b, b.k);
        d.s0 = f32(b.roughness * b.roughness);
        break;
    case BasicKind::Dielectric:
        d.s0 = f32(b.roughness * b.roughness);
        d.s1 = f32(b.ior);
        break;
    }
    return d;
}

void putAffine(float* out, const Affine& map)
{
    for (int row{0}; row < 3; ++row) {
        out[4 * row + 0] = f32(map.linear[row][0]);
        out[4 * row + 1] = f32(map.linear[row][1]);
        out[4 * row + 2] = f32(map.linear[row][2]);
    }
    out[3] = f32(map.offset.x);
    out[7] = f32(map.offset.y);
    out[11] = f32(map.offset.z);
}

// Spheres whose coordinates reach 256 need the FP64 quadratic: beyond that,
// FP32 resolves o - c only to about 1.5e-5 and |o - c|^2 - r^2 cancels.
bool needsWideSphere(const SphereDesc& s)
{
    const double extent{std::max({std::abs(s.center.x), std::abs(s.center.y), std::abs(s.center.z)}) + s.radius};
    return extent >= 256.0;
}

} // namespace

DeviceImage flattenScene(const HostScene& scene)
{
    DeviceImage image;

    // Scene triangles (objects of kind Triangle) occupy the start of the
    // triangle table in add order; each mesh's triangles follow in leaf order.
    for (std::size_t i{0}; i < scene.triangles.size(); ++i) {
        image.triangles.push_back(deviceTriangle(scene.triangles[i], static_cast<std::uint32_t>(i)));
        image.attrs.push_back(deviceAttr(scene.triangles[i], nullptr));
    }
    std::vector<std::uint32_t> mesh_root(scene.meshes.size(), kEmptyChild);
    std::uint32_t max_blas_depth{0};
    for (std::size_t m{0}; m < scene.meshes.size(); ++m) {
        const MeshDesc& mesh{scene.meshes[m]};
        const std::uint64_t base{image.triangles.size()};
        image.mesh_triangle_base.push_back(static_cast<std::uint32_t>(base));
        for (const std::uint32_t t : mesh.bvh.order) {
            image.triangles.push_back(deviceTriangle(mesh.triangles[t], t));
            image.attrs.push_back(deviceAttr(mesh.triangles[t], mesh.corner_normals.empty() ? nullptr : &mesh.corner_normals[t]));
        }
        mesh_root[m] = emitBvh(mesh.bvh, base, image.nodes);
        max_blas_depth = std::max(max_blas_depth, mesh.bvh.max_depth);
    }
    if (image.triangles.size() > kMaxLeafFirst) {
        throw std::invalid_argument{std::format("scene has more than {} triangles", kMaxLeafFirst)};
    }

    image.tlas_root = emitBvh(scene.tlas, 0, image.nodes);
    image.stack_need = scene.tlas.max_depth + max_blas_depth + 3;

    image.object_position.assign(scene.objects.size(), 0);
    for (std::size_t pos{0}; pos < scene.tlas.order.size(); ++pos) {
        const std::uint32_t id{scene.tlas.order[pos]};
        const ObjectDesc& object{scene.objects[id]};
        DevObject d{};
        d.id = id;
        d.material = object.material;
        switch (object.kind) {
        case ObjectKind::Sphere:
            d.kind = needsWideSphere(scene.spheres[object.index]) ? kObjSphereWide : kObjSphere;
            d.index = object.index;
            break;
        case ObjectKind::Triangle:
            d.kind = kObjTriangle;
            d.index = object.index;
            break;
        case ObjectKind::Instance:
            d.kind = kObjInstance;
            d.index = object.index;
            break;
        }
        image.objects.push_back(d);
        image.object_position[id] = static_cast<std::uint32_t>(pos);
    }
    image.object_light.resize(scene.objects.size());
    for (std::size_t id{0}; id < scene.objects.size(); ++id) {
        image.object_light[id] = scene.objects[id].light;
    }

    for (const SphereDesc& s : scene.spheres) {
        image.spheres.push_back({f32(s.center.x), f32(s.center.y), f32(s.center.z), f32(s.radius)});
    }
    for (const InstanceDesc& inst : scene.instances) {
        DevInstance d{};
        putAffine(d.to_object, inst.to_object.forward());
        putAffine(d.to_world, inst.to_world.forward());
        d.root = mesh_root[inst.mesh];
        d.mesh = inst.mesh;
        image.instances.push_back(d);
        const Affine& back{inst.to_object.forward()};
        for (int row{0}; row < 3; ++row) {
            image.instance_to_object64.push_back(back.linear[row][0]);
            image.instance_to_object64.push_back(back.linear[row][1]);
            image.instance_to_object64.push_back(back.linear[row][2]);
            image.instance_to_object64.push_back(row == 0 ? back.offset.x : (row == 1 ? back.offset.y : back.offset.z));
        }
    }
    for (const MaterialDesc& m : scene.materials) {
        DevMaterial d{};
        d.mix = m.mix ? 1u : 0u;
        d.scale = f32(m.scale);
        d.veins = f32(m.veins);
        d.threshold = f32(m.threshold);
        d.first = deviceBasic(m.first);
        d.second = deviceBasic(m.mix ? m.second : m.first);
        image.materials.push_back(d);
    }
    if (image.materials.empty()) {
        image.materials.push_back(DevMaterial{});
    }
    for (const LightDesc& l : scene.lights) {
        DevLight d{};
        d.kind = static_cast<std::uint32_t>(l.kind);
        d.object = l.kind == LightKind::Area ? image.object_position[l.object] : 0xFFFFFFFFu;
        d.radius = f32(l.radius);
        d.p[0] = f32(l.position.x);
        d.p[1] = f32(l.position.y);
        d.p[2] = f32(l.position.z);
        if (l.kind == LightKind::Sky) {
            putRgb(d.e, l.nadir);
            putRgb(d.z, l.zenith);
        } else {
            putRgb(d.e, l.emission);
        }
        image.lights.push_back(d);
    }
    image.sky_light = scene.sky_light;
    return image;
}

DevCamera deviceCamera(const HostScene& scene, int width, int height)
{
    const CameraFrame frame{scene.cameraFrame(static_cast<double>(width) / static_cast<double>(height))};
    DevCamera cam{};
    const auto put = [](float* out, Vec3 v) {
        out[0] = f32(v.x);
        out[1] = f32(v.y);
        out[2] = f32(v.z);
    };
    put(cam.origin, frame.origin);
    put(cam.forward, frame.forward);
    put(cam.half_width, frame.half_width);
    put(cam.half_height, frame.half_height);
    return cam;
}

} // namespace albedo_b200
