// Flattening: the reference-topology BVHs become child-box nodes over FP32 boxes
// rounded outward; primitives are stored in leaf order so a leaf is one
// contiguous run; everything else becomes flat FP32 tables.
#include "flatten.hpp"

#include <algorithm>
#include <array>
#include <bit>
#include <cmath>
#include <format>
#include <stdexcept>
#include <thread>
#include <vector>

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
    node.lo_x[child] = roundDown(box.min.x);
    node.hi_x[child] = roundUp(box.max.x);
    node.lo_y[child] = roundDown(box.min.y);
    node.hi_y[child] = roundUp(box.max.y);
    node.lo_z[child] = roundDown(box.min.z);
    node.hi_z[child] = roundUp(box.max.z);
}

struct Emitted {
    std::uint32_t root{kEmptyChild};
    // Most traversal-stack entries a query over this tree can hold at once.
    std::uint32_t stack_need{0};
};

// Emits `bvh` (binary, depth-first, first child at i + 1) as 4-wide nodes, each
// collapsing an interior node and its interior children. Leaves index
// primitives from `prim_base` in leaf order. For every ray octant the node lists
// its children in the order the reference's traversal (accel/bvh.hpp:239-278,
// near child by the sign of the split axis) reaches them, so the order in which
// leaves are visited is the reference's. A root that is a leaf gets a node with
// that one child.
Emitted emitBvh(const BuiltBvh& bvh, std::uint64_t prim_base, std::vector<DevNode>& out)
{
    Emitted emitted;
    if (bvh.nodes.empty()) {
        return emitted;
    }
    const auto isLeaf = [&](std::size_t i) { return bvh.nodes[i].count != 0; };
    const auto secondOf = [&](std::size_t i) { return static_cast<std::size_t>(bvh.nodes[i].offset); };
    // Binary nodes that head a 4-wide node, and the 4-wide index of each.
    std::vector<std::uint32_t> device_index(bvh.nodes.size(), kEmptyChild);
    std::vector<std::size_t> heads{0};
    device_index[0] = static_cast<std::uint32_t>(out.size());
    out.emplace_back();
    std::vector<std::uint32_t> need(bvh.nodes.size(), 0);
    // Heads are discovered in order; their children are filled afterwards.
    for (std::size_t h{0}; h < heads.size(); ++h) {
        const std::size_t i{heads[h]};
        std::array<std::size_t, 4> slots{};
        std::size_t used{0};
        if (isLeaf(i)) {
            slots[used++] = i;
        } else {
            for (const std::size_t x : {i + 1, secondOf(i)}) {
                if (isLeaf(x)) {
                    slots[used++] = x;
                } else {
                    slots[used++] = x + 1;
                    slots[used++] = secondOf(x);
                }
            }
        }
        for (std::size_t k{0}; k < used; ++k) {
            const std::size_t s{slots[k]};
            if (!isLeaf(s) && device_index[s] == kEmptyChild) {
                device_index[s] = static_cast<std::uint32_t>(out.size());
                out.emplace_back();
                heads.push_back(s);
            }
        }
    }
    // Fill nodes bottom-up (heads in reverse discovery order) so stack needs of
    // children are known when their parent is filled.
    for (std::size_t h{heads.size()}; h-- > 0;) {
        const std::size_t i{heads[h]};
        DevNode& dev{out[device_index[i]]};
        dev = DevNode{};
        for (int c{0}; c < 4; ++c) {
            dev.child[c] = kEmptyChild;
        }
        if (isLeaf(i)) {
            setChildBox(dev, 0, bvh.nodes[i].bounds);
            dev.child[0] = leafRef(prim_base + bvh.nodes[i].offset, bvh.nodes[i].count);
            dev.count = 1;
            continue;
        }
        // Groups: the first and second child of i, each a leaf or two children.
        struct Group {
            std::size_t node;
            int first_slot;
            int size;
        };
        std::array<Group, 2> groups{};
        int slot{0};
        const std::array<std::size_t, 2> halves{i + 1, secondOf(i)};
        for (int g{0}; g < 2; ++g) {
            const std::size_t x{halves[g]};
            groups[g] = {x, slot, isLeaf(x) ? 1 : 2};
            const std::array<std::size_t, 2> kids{x + 1, isLeaf(x) ? 0 : secondOf(x)};
            for (int k{0}; k < groups[g].size; ++k) {
                const std::size_t s{isLeaf(x) ? x : kids[k]};
                setChildBox(dev, slot, bvh.nodes[s].bounds);
                dev.child[slot] = isLeaf(s) ? leafRef(prim_base + bvh.nodes[s].offset, bvh.nodes[s].count)
                                            : device_index[s];
                ++slot;
            }
        }
        dev.count = static_cast<std::uint32_t>(slot);
        // The binary structure this node collapses, for counting the boxes the
        // reference's traversal tests: group g holds the first or second child of
        // node i (1 slot if a leaf, else its 2 children).
        dev.groups = static_cast<std::uint32_t>(groups[0].size) | (static_cast<std::uint32_t>(groups[1].size) << 2U);
        for (unsigned octant{0}; octant < 8; ++octant) {
            const bool swap{((octant >> bvh.nodes[i].axis) & 1U) != 0};
            std::uint8_t packed{0};
            int position{0};
            for (int g{0}; g < 2; ++g) {
                const Group& group{groups[swap ? 1 - g : g]};
                if (group.size == 1) {
                    packed |= static_cast<std::uint8_t>(group.first_slot << (2 * position++));
                } else {
                    const bool inner_swap{((octant >> bvh.nodes[group.node].axis) & 1U) != 0};
                    packed |= static_cast<std::uint8_t>((group.first_slot + (inner_swap ? 1 : 0)) << (2 * position++));
                    packed |= static_cast<std::uint8_t>((group.first_slot + (inner_swap ? 0 : 1)) << (2 * position++));
                }
            }
            dev.order[octant] = packed;
        }
        // Stack need: pushes here (count - 1) plus the deepest interior child's need.
        std::uint32_t child_need{0};
        for (int g{0}; g < 2; ++g) {
            const std::size_t x{halves[g]};
            const std::array<std::size_t, 2> kids{x + 1, isLeaf(x) ? 0 : secondOf(x)};
            for (int k{0}; k < groups[g].size; ++k) {
                const std::size_t s{isLeaf(x) ? x : kids[k]};
                if (!isLeaf(s)) {
                    child_need = std::max(child_need, need[s]);
                }
            }
        }
        need[i] = dev.count - 1 + child_need;
    }
    emitted.root = device_index[0];
    emitted.stack_need = need[0];
    return emitted;
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

bool allFinite(const float* v, std::size_t n)
{
    for (std::size_t i{0}; i < n; ++i) {
        if (!std::isfinite(v[i])) {
            return false;
        }
    }
    return true;
}

// The reference stores geometry in FP64; the device tables hold FP32, so a
// value beyond FP32's range (about 3.4e38) would become infinite there.
void checkFp32Range(const DeviceImage& image)
{
    const auto fail = [](const char* what, std::size_t index) {
        throw LayoutLimitError{std::format("{} {} has a coordinate beyond the FP32 range of the device tables "
                                           "(magnitude above 3.4e38)",
                                           what, index)};
    };
    for (std::size_t i{0}; i < image.spheres.size(); ++i) {
        const DevSphere& s{image.spheres[i]};
        const float v[4]{s.cx, s.cy, s.cz, s.r};
        if (!allFinite(v, 4)) {
            fail("sphere", i);
        }
    }
    for (std::size_t i{0}; i < image.triangles.size(); ++i) {
        const DevTriangle& t{image.triangles[i]};
        const float v[9]{t.v0x, t.v0y, t.v0z, t.v1x, t.v1y, t.v1z, t.v2x, t.v2y, t.v2z};
        if (!allFinite(v, 9)) {
            fail("triangle", i);
        }
    }
    for (std::size_t i{0}; i < image.instances.size(); ++i) {
        if (!allFinite(image.instances[i].to_object, 12) || !allFinite(image.instances[i].to_world, 12)) {
            fail("instance", i);
        }
    }
    for (std::size_t i{0}; i < image.lights.size(); ++i) {
        const DevLight& l{image.lights[i]};
        const float v[4]{l.p[0], l.p[1], l.p[2], l.radius};
        if (!allFinite(v, 4)) {
            fail("light", i);
        }
    }
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
    std::uint32_t max_blas_need{0};
    for (std::size_t m{0}; m < scene.meshes.size(); ++m) {
        const MeshDesc& mesh{scene.meshes[m]};
        const std::uint64_t base{image.triangles.size()};
        image.mesh_triangle_base.push_back(static_cast<std::uint32_t>(base));
        // Each triangle converts on its own, so large meshes convert in chunks
        // on several threads.
        const std::size_t count{mesh.bvh.order.size()};
        image.triangles.resize(base + count);
        image.attrs.resize(base + count);
        const std::size_t chunks{count < (std::size_t{1} << 16)
                                     ? 1
                                     : std::max<std::size_t>(1, std::thread::hardware_concurrency())};
        // A jthread joins when destroyed, so an exception that leaves early (a
        // thread that fails to start, or the calling thread's own share) still
        // waits for the workers already running.
        std::vector<std::jthread> workers;
        const auto convert = [&](std::size_t chunk) {
            for (std::size_t pos{count * chunk / chunks}; pos < count * (chunk + 1) / chunks; ++pos) {
                const std::uint32_t t{mesh.bvh.order[pos]};
                image.triangles[base + pos] = deviceTriangle(mesh.triangles[t], t);
                image.attrs[base + pos] =
                    deviceAttr(mesh.triangles[t], mesh.corner_normals.empty() ? nullptr : &mesh.corner_normals[t]);
            }
        };
        for (std::size_t chunk{1}; chunk < chunks; ++chunk) {
            workers.emplace_back(convert, chunk);
        }
        convert(0);
        for (std::jthread& worker : workers) {
            worker.join();
        }
        const Emitted blas{emitBvh(mesh.bvh, base, image.nodes)};
        mesh_root[m] = blas.root;
        max_blas_need = std::max(max_blas_need, blas.stack_need);
    }
    if (image.triangles.size() > kMaxLeafFirst) {
        throw std::invalid_argument{std::format("scene has more than {} triangles", kMaxLeafFirst)};
    }

    const Emitted tlas{emitBvh(scene.tlas, 0, image.nodes)};
    image.tlas_root = tlas.root;
    // TLAS pushes, then a resume entry and an exit marker when entering an
    // instance, then the deepest BLAS's pushes.
    image.stack_need = tlas.stack_need + 2 + max_blas_need;

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
    checkFp32Range(image);
    return image;
}

DevCamera deviceCamera(const HostScene& scene, int width, int height)
{
    return deviceCamera(scene.camera, width, height);
}

DevCamera deviceCamera(const CameraSettings& settings, int width, int height)
{
    const CameraFrame frame{buildCameraFrame(settings, static_cast<double>(width) / static_cast<double>(height))};
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
    if (!allFinite(cam.origin, 3) || !allFinite(cam.forward, 3) || !allFinite(cam.half_width, 3) ||
        !allFinite(cam.half_height, 3)) {
        throw LayoutLimitError{"the camera has a coordinate beyond the FP32 range of the device"};
    }
    return cam;
}

} // namespace albedo_b200
