// Ray queries over the two-level BVH: TLAS over objects, BLAS per shared mesh.
//
// Restates, in FP32 over the device layout, the reference's query path:
//   Bvh::traverse / nearestHit / anyHit   accel/bvh.hpp:211-267
//   clipToSlab with Ize's exit widening    accel/bvh.hpp:80-103
//   orderedChildren (near child by sign)   accel/bvh.hpp:118-129
//   Sphere::intersect (Haines)             geometry/sphere.cpp:92-135
//   Triangle::intersect (watertight)       geometry/triangle.cpp:132-176
//   MeshInstance::intersect                geometry/mesh_instance.cpp:32-48
// The node order, the near/far rule and "a later hit must be strictly nearer"
// are the reference's, so ties resolve the same way. Boxes are FP32 rounded
// outward, which can only add box hits, never lose one.
//
// The traversal stack lives in shared memory: entry i of thread `lane` is at
// stack[i * stride + lane] (entry-major, so a warp touching the same depth hits
// consecutive banks). An entry is either (child reference, entry distance), 8
// bytes, and a popped entry whose box is entered beyond the current hit is
// dropped as the reference drops it; or the child reference alone, 4 bytes,
// and the popped node or leaf is visited and culled by its own box tests. Both
// give the same hits: a primitive below a node entered beyond the current hit
// cannot be hit nearer than it. The 4-byte form halves the shared memory of
// the wavefront's persistent traversal kernels, so more of them fit on an SM.
#pragma once

#include "common.cuh"

namespace albedo_b200 {

// 1 + 2 gamma(3) for FP32 (u = 2^-24), rounded up: Ize 2013 as in accel/bvh.hpp:80-84.
constexpr float kBoxExitWidening = 1.00000036f;
constexpr std::uint32_t kExitMarker = 0x7FFFFFFFu; // stack entry: leave the current instance
constexpr std::uint32_t kNoPrim = 0xFFFFFFFFu;

enum SphereSkip : int { kSphereTestBoth = 0, kSphereSkipAll = 1, kSphereFarOnly = 2 };

// What a ray leaving a surface must not hit again. A triangle cannot be hit
// again by a ray leaving it; a sphere left outward cannot be hit again, and one
// left inward only at its far root. This replaces the reference's FP64-scale
// 1e-7 origin offset (estimator/surface_ray.hpp:18-31), which FP32 cannot
// resolve, with the exact statement it approximates.
struct SkipRule {
    std::uint32_t object_pos;  // TLAS leaf position of the object left, or kNoPrim
    std::uint32_t tri_pos;     // triangle table position left (instances), or kNoPrim
    int sphere_mode;           // SphereSkip for a sphere object
    std::uint32_t light_object_pos; // shadow rays: the area light's own object, or kNoPrim

    ALB_DEV static SkipRule none() { return {kNoPrim, kNoPrim, kSphereTestBoth, kNoPrim}; }
};

// Work one query did, for the algorithmic-bytes figure: child boxes tested,
// triangles and spheres tested, instances entered, queries traced, and the
// boxes the reference's binary traversal tests for the same query (one per node
// it pops, accel/bvh.hpp:239-278).
struct TraversalCounts {
    unsigned long long boxes;
    unsigned long long triangles;
    unsigned long long spheres;
    unsigned long long instances;
    unsigned long long rays;
    unsigned long long reference_boxes;
};

struct TraceHit {
    float t;
    std::uint32_t obj_pos; // TLAS leaf position of the object hit
    std::uint32_t tri_pos; // triangle table position, or kNoPrim for spheres
    float b0, b1, b2;      // barycentric weights of a triangle hit
};

// The ray as traversal and the watertight test need it (accel/bvh.hpp:60-78,
// geometry/triangle.cpp:81-106).
struct TravRay {
    float3 o, inv; // the direction itself is the caller's (spheres, the only users, are in world space)
    std::uint32_t neg; // bit a set when d[a] < 0
    int kx, ky, kz;
    float sx, sy, sz;
    std::uint32_t planes; // bit a set when inv[a] is negative (-0 directions included): the box test's near planes
    bool usable;          // |d|^2 is a normal number

    ALB_DEV void setup(float3 origin, float3 dir)
    {
        o = origin;
        inv = mk(1.0f / dir.x, 1.0f / dir.y, 1.0f / dir.z);
        neg = (dir.x < 0.0f ? 1u : 0u) | (dir.y < 0.0f ? 2u : 0u) | (dir.z < 0.0f ? 4u : 0u);
        planes = (signbit(inv.x) ? 1u : 0u) | (signbit(inv.y) ? 2u : 0u) | (signbit(inv.z) ? 4u : 0u);
        usable = isNormalF(lengthSquared(dir));
        const float mx = fabsf(dir.x);
        const float my = fabsf(dir.y);
        const float mz = fabsf(dir.z);
        kz = mx > my ? (mx > mz ? 0 : 2) : (my > mz ? 1 : 2);
        kx = kz == 2 ? 0 : kz + 1;
        ky = kx == 2 ? 0 : kx + 1;
        const float dz = comp(dir, kz);
        if (dz < 0.0f) {
            const int t = kx;
            kx = ky;
            ky = t;
        }
        sx = comp(dir, kx) / dz;
        sy = comp(dir, ky) / dz;
        sz = 1.0f / dz;
    }
};

// clipToSlab on all three axes for one box; returns whether [tmin, tmax]
// survives and the clipped entry distance (accel/bvh.hpp:93-114).
ALB_DEV bool slabTest(float lox, float hix, float loy, float hiy, float loz, float hiz, const TravRay& r, float tmin,
                      float tmax, float& entry)
{
    float lo = tmin;
    float hi = tmax;
    float n, f;
#define ALB_CLIP(LO, HI, O, INV)                                                                                       \
    n = ((LO) - (O)) * (INV);                                                                                          \
    f = ((HI) - (O)) * (INV);                                                                                          \
    if (n > f) {                                                                                                       \
        const float s_ = n;                                                                                            \
        n = f;                                                                                                         \
        f = s_;                                                                                                        \
    }                                                                                                                  \
    f *= f < 0.0f ? 2.0f - kBoxExitWidening : kBoxExitWidening;                                                        \
    lo = n > lo ? n : lo;                                                                                              \
    hi = f < hi ? f : hi;
    ALB_CLIP(lox, hix, r.o.x, r.inv.x)
    ALB_CLIP(loy, hiy, r.o.y, r.inv.y)
    ALB_CLIP(loz, hiz, r.o.z, r.inv.z)
#undef ALB_CLIP
    entry = lo;
    return lo <= hi;
}

// Three-input FP32 maximum and minimum (one instruction each on sm_100a). A NaN
// operand is skipped as the two-input fmaxf/fminf chain skips it (checked on a
// B200 against that chain over every triple of NaN, infinities, signed zeros,
// a subnormal and ordinary values).
__device__ __forceinline__ float max3f(float a, float b, float c)
{
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float min3f(float a, float b, float c)
{
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// slabTest without branches, given the box's near and far planes on each axis:
// lo and hi where the inverse direction's sign bit is clear, hi and lo where it
// is set (a -0 direction component gives a -infinite inverse, so it counts as
// negative). It returns slabTest's answer and entry distance (up to the sign of
// a zero entry distance, which only comparisons read):
//   - With a finite nonzero inverse no distance is NaN, and rounding is
//     monotone, so (near - o) * inv <= (far - o) * inv: these are the clip's
//     entry and exit distances after its swap.
//   - The entry is the largest of tmin and the three axis entries, in any order;
//     the three-input maximum and minimum skip a NaN operand as the clip's
//     comparisons do.
//   - The exit widening w(f) = f * (f < 0 ? 2 - W : W) is nondecreasing, so
//     min(tmax, w(fx), w(fy), w(fz)) = min(tmax, w(min(fx, fy, fz))); and
//     w(f) = max(f * W, f * (2 - W)) since W > 1.
//   - An infinite inverse (a zero or subnormal direction component) gives the
//     clip's answer on that axis too, with one exception: for a -infinite
//     inverse and an origin lying exactly on one of the slab's two planes (not
//     both), the clip's NaN, left in place by its swap rule, rejects the box
//     (or, over an unbounded range, enters it at +infinity), and this test
//     enters it at the other axes' entry. Entering a box more can only add
//     primitive tests, never lose a hit. (Checked on the host over 8 M rays,
//     tests/cpp/box_test.cpp.)
// The four children of a node test independently.
__device__ __forceinline__ bool slabTestOrdered(float nx, float fx, float ny, float fy, float nz, float fz,
                                                const TravRay& r, float tmin, float tmax, float& entry)
{
    const float tnx = __fmul_rn(__fsub_rn(nx, r.o.x), r.inv.x);
    const float tfx = __fmul_rn(__fsub_rn(fx, r.o.x), r.inv.x);
    const float tny = __fmul_rn(__fsub_rn(ny, r.o.y), r.inv.y);
    const float tfy = __fmul_rn(__fsub_rn(fy, r.o.y), r.inv.y);
    const float tnz = __fmul_rn(__fsub_rn(nz, r.o.z), r.inv.z);
    const float tfz = __fmul_rn(__fsub_rn(fz, r.o.z), r.inv.z);
    const float lo = max3f(tnx, tny, fmaxf(tnz, tmin));
    const float f = min3f(tfx, tfy, tfz);
    const float hi = fminf(fmaxf(__fmul_rn(f, kBoxExitWidening), __fmul_rn(f, 2.0f - kBoxExitWidening)), tmax);
    entry = lo;
    return lo <= hi;
}

// Explicitly rounded arithmetic: every product and sum rounds on its own, as the
// reference (built without contraction) rounds in FP64. Traversal code uses them
// so that every kernel compiles a query to the same operations: an FMA the
// compiler may contract in one kernel and not in another would give two kernels
// different hit distances.
ALB_DEV float rmul(float a, float b) { return __fmul_rn(a, b); }
ALB_DEV float radd(float a, float b) { return __fadd_rn(a, b); }
ALB_DEV float rsub(float a, float b) { return __fsub_rn(a, b); }
ALB_DEV double rmul(double a, double b) { return __dmul_rn(a, b); }
ALB_DEV double radd(double a, double b) { return __dadd_rn(a, b); }
ALB_DEV double rsub(double a, double b) { return __dsub_rn(a, b); }
template <typename T>
ALB_DEV T rdot(T ax, T ay, T az, T bx, T by, T bz)
{
    return radd(radd(rmul(ax, bx), rmul(ay, by)), rmul(az, bz));
}

// Haines' sphere test in precision T (geometry/sphere.cpp:92-135), returning the
// nearest root strictly inside (tmin, tmax), honouring the skip mode.
template <typename T>
ALB_DEV bool sphereRoot(T ox, T oy, T oz, T dx, T dy, T dz, T cx, T cy, T cz, T radius, T tmin, T tmax, int mode,
                        T& t_out)
{
    const T ocx = rsub(ox, cx);
    const T ocy = rsub(oy, cy);
    const T ocz = rsub(oz, cz);
    const T a = rdot(dx, dy, dz, dx, dy, dz);
    const T h = rdot(dx, dy, dz, ocx, ocy, ocz);
    const T r2 = rmul(radius, radius);
    const T c = rsub(rdot(ocx, ocy, ocz, ocx, ocy, ocz), r2);
    const T k = h / a;
    const T lx = rsub(ocx, rmul(dx, k));
    const T ly = rsub(ocy, rmul(dy, k));
    const T lz = rsub(ocz, rmul(dz, k));
    const T disc = rmul(a, rsub(r2, rdot(lx, ly, lz, lx, ly, lz)));
    if (disc < T(0)) {
        return false;
    }
    const T q = -radd(h, copysign(sqrt(disc), h));
    T near_root = T(0);
    T far_root = T(0);
    if (q != T(0)) {
        near_root = q / a;
        far_root = c / q;
        if (near_root > far_root) {
            const T s = near_root;
            near_root = far_root;
            far_root = s;
        }
    }
    T t = near_root;
    if (mode == kSphereFarOnly || !(tmin < t && t < tmax)) {
        t = far_root;
        if (!(tmin < t && t < tmax)) {
            return false;
        }
    }
    // A hit point that rounds onto the center has no normal: a miss (geometry/sphere.cpp:121-126).
    const T px = rsub(radd(ox, rmul(dx, t)), cx);
    const T py = rsub(radd(oy, rmul(dy, t)), cy);
    const T pz = rsub(radd(oz, rmul(dz, t)), cz);
    if (!(rdot(px, py, pz, px, py, pz) > T(0))) {
        return false;
    }
    t_out = t;
    return true;
}

// `r` is the world-space ray whose direction is `d`.
ALB_DEV bool intersectSphere(const TravRay& r, float3 d, const DevSphere& s, bool wide, float tmin, float tmax,
                             int mode, float& t)
{
    if (!r.usable) {
        return false;
    }
    if (wide) {
        // Coordinates of order 1e4 (room-sized walls): o - c and |o - c|^2 - r^2
        // cancel catastrophically in FP32, so the quadratic runs in FP64.
        double td;
        if (!sphereRoot<double>(r.o.x, r.o.y, r.o.z, d.x, d.y, d.z, s.cx, s.cy, s.cz, s.r, tmin, tmax, mode, td)) {
            return false;
        }
        const float tf = static_cast<float>(td);
        if (!(tmin < tf && tf < tmax)) {
            return false;
        }
        t = tf;
        return true;
    }
    return sphereRoot<float>(r.o.x, r.o.y, r.o.z, d.x, d.y, d.z, s.cx, s.cy, s.cz, s.r, tmin, tmax, mode, t);
}

// Woop-Benthin-Wald watertight test (geometry/triangle.cpp:132-176). Every
// product is rounded on its own (no FMA), so edge functions of triangles sharing
// an edge are exact negations; zero edge functions are recomputed in FP64.
ALB_DEV bool intersectTriangle(const TravRay& r, const float4& p0, const float4& p1, const float4& p2, float tmin,
                               float tmax, float& t, float& b0, float& b1, float& b2)
{
    const float3 A = mk(__fsub_rn(p0.x, r.o.x), __fsub_rn(p0.y, r.o.y), __fsub_rn(p0.z, r.o.z));
    const float3 B = mk(__fsub_rn(p1.x, r.o.x), __fsub_rn(p1.y, r.o.y), __fsub_rn(p1.z, r.o.z));
    const float3 C = mk(__fsub_rn(p2.x, r.o.x), __fsub_rn(p2.y, r.o.y), __fsub_rn(p2.z, r.o.z));
    const float az = comp(A, r.kz);
    const float bz = comp(B, r.kz);
    const float cz = comp(C, r.kz);
    const float ax = __fsub_rn(comp(A, r.kx), __fmul_rn(r.sx, az));
    const float ay = __fsub_rn(comp(A, r.ky), __fmul_rn(r.sy, az));
    const float bx = __fsub_rn(comp(B, r.kx), __fmul_rn(r.sx, bz));
    const float by = __fsub_rn(comp(B, r.ky), __fmul_rn(r.sy, bz));
    const float cx = __fsub_rn(comp(C, r.kx), __fmul_rn(r.sx, cz));
    const float cy = __fsub_rn(comp(C, r.ky), __fmul_rn(r.sy, cz));
    float u = __fsub_rn(__fmul_rn(cx, by), __fmul_rn(cy, bx));
    float v = __fsub_rn(__fmul_rn(ax, cy), __fmul_rn(ay, cx));
    float w = __fsub_rn(__fmul_rn(bx, ay), __fmul_rn(by, ax));
    if (u == 0.0f || v == 0.0f || w == 0.0f) {
        const double du = static_cast<double>(cx) * by - static_cast<double>(cy) * bx;
        const double dv = static_cast<double>(ax) * cy - static_cast<double>(ay) * cx;
        const double dw = static_cast<double>(bx) * ay - static_cast<double>(by) * ax;
        u = static_cast<float>(du);
        v = static_cast<float>(dv);
        w = static_cast<float>(dw);
    }
    const bool inside = (u >= 0.0f && v >= 0.0f && w >= 0.0f) || (u <= 0.0f && v <= 0.0f && w <= 0.0f);
    if (!inside) {
        return false;
    }
    const float det = __fadd_rn(__fadd_rn(u, v), w);
    if (det == 0.0f) {
        return false;
    }
    const float tz = __fadd_rn(__fadd_rn(__fmul_rn(u, __fmul_rn(r.sz, az)), __fmul_rn(v, __fmul_rn(r.sz, bz))),
                               __fmul_rn(w, __fmul_rn(r.sz, cz)));
    const float tt = __fdiv_rn(tz, det);
    if (!(tmin < tt && tt < tmax)) {
        return false;
    }
    t = tt;
    b0 = __fdiv_rn(u, det);
    b1 = __fdiv_rn(v, det);
    b2 = __fdiv_rn(w, det);
    return true;
}

// An instance's 3x4 row-major affine map applied to a point and to a vector,
// explicitly rounded (the ray a query carries into an instance must be the
// same in every kernel).
ALB_DEV float3 affinePoint(const float* m, float3 p)
{
    return mk(radd(rdot(m[0], m[1], m[2], p.x, p.y, p.z), m[3]), radd(rdot(m[4], m[5], m[6], p.x, p.y, p.z), m[7]),
              radd(rdot(m[8], m[9], m[10], p.x, p.y, p.z), m[11]));
}
ALB_DEV float3 affineVector(const float* m, float3 v)
{
    return mk(rdot(m[0], m[1], m[2], v.x, v.y, v.z), rdot(m[4], m[5], m[6], v.x, v.y, v.z),
              rdot(m[8], m[9], m[10], v.x, v.y, v.z));
}
// Transpose of the linear part times v: how a normal maps under the inverse map.
ALB_DEV float3 affineTransposedVector(const float* m, float3 v)
{
    return mk(m[0] * v.x + m[4] * v.y + m[8] * v.z, m[1] * v.x + m[5] * v.y + m[9] * v.z,
              m[2] * v.x + m[6] * v.y + m[10] * v.z);
}

ALB_DEV std::uint32_t leafRef(std::uint32_t first, std::uint32_t count)
{
    return kLeafBit | ((count - 1u) << 28) | first;
}

// One ray query in flight: the ray in the space being traversed (world or the
// current instance's object space), the world ray it came from, the live range,
// the node reference to visit next, the stack depth and the hit so far.
struct TraceState {
    TravRay r;
    float3 origin;
    float3 dir;
    float tmin;
    float tmax;
    std::uint32_t ref;
    std::uint32_t inst_pos; // TLAS leaf position of the instance being traversed, or kNoPrim
    int sp;
    bool found;
    // The ray changes space (entering or leaving an instance): r.o and r.inv
    // hold the new origin and direction, and the next step sets the ray up from
    // them. One set-up site keeps the traversal's code small.
    bool resetup;
    TraceHit hit;

    ALB_DEV void changeSpace(float3 o, float3 d)
    {
        r.o = o;
        r.inv = d;
        resetup = true;
    }
    ALB_DEV void settle()
    {
        if (resetup) {
            r.setup(r.o, r.inv);
            resetup = false;
        }
    }
};

// What a traversal step leaves to do next.
enum TraceStep : int {
    kStepDescend = 0, // `ref` holds the next node or leaf to visit
    kStepPop = 1,     // continue with the next stack entry
    kStepFinished = 2 // any-hit found, or the stack would overflow (error flag set)
};

// Starts a query over (tmin, tmax); false when the scene has no objects.
ALB_DEV bool traceBegin(const DevScene& s, TraceState& q, float3 origin, float3 dir, float tmin, float tmax)
{
    q.origin = origin;
    q.dir = dir;
    q.tmin = tmin;
    q.tmax = tmax;
    q.found = false;
    q.resetup = false;
    q.sp = 0;
    q.inst_pos = kNoPrim;
    q.ref = s.tlas_root;
    if (s.tlas_root == kEmptyChild) {
        return false;
    }
    q.r.setup(origin, dir);
    return true;
}

// The boxes the reference's binary traversal tests below a 4-wide node: it pops
// both binary children (one box each) and, for a binary child that is interior
// and whose box the ray enters, both of its children. That child's box is the
// union of the two slots it became.
__device__ __forceinline__ float slotOf(const float4& v, int k)
{
    return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}

__device__ __forceinline__ void countReferenceBoxes(const float4& lx, const float4& hx, const float4& ly,
                                                    const float4& hy, const float4& lz, const float4& hz,
                                                    unsigned groups, const TravRay& r, float tmin, float tmax,
                                                    TraversalCounts& counts)
{
    if (groups == 0u) {
        return;
    }
    counts.reference_boxes += 2;
    int first = 0;
    for (int g = 0; g < 2; ++g) {
        const int size = static_cast<int>((groups >> (2 * g)) & 3u);
        if (size == 2) {
            const int a = first;
            const int b = first + 1;
            float entry;
            if (slabTest(fminf(slotOf(lx, a), slotOf(lx, b)), fmaxf(slotOf(hx, a), slotOf(hx, b)),
                         fminf(slotOf(ly, a), slotOf(ly, b)), fmaxf(slotOf(hy, a), slotOf(hy, b)),
                         fminf(slotOf(lz, a), slotOf(lz, b)), fmaxf(slotOf(hz, a), slotOf(hz, b)), r, tmin, tmax,
                         entry)) {
                counts.reference_boxes += 2;
            }
        }
        first += size;
    }
}

// One stack entry: child reference and entry distance, or the reference alone.
__device__ __forceinline__ void pushEntry(uint2* slot, std::uint32_t ref, float entry)
{
    *slot = make_uint2(ref, __float_as_uint(entry));
}
__device__ __forceinline__ void pushEntry(unsigned* slot, std::uint32_t ref, float)
{
    *slot = ref;
}

// A 4-wide node: tests every child box, continues with the hit child the
// reference reaches first and pushes the other hit children, last first, so
// leaves are reached in the reference's depth-first near-first order.
template <typename Stack>
__device__ __forceinline__ int nodeStep(const DevNode* nodes, TraceState& q, Stack* stack, int stride,
                                        int stack_size, unsigned int* error_flag, TraversalCounts* counts)
{
    const float4* np = reinterpret_cast<const float4*>(nodes + q.ref);
    const uint4 ch = __ldg(reinterpret_cast<const uint4*>(np + 6));
    const uint4 meta = __ldg(reinterpret_cast<const uint4*>(np + 7));
    const int present = static_cast<int>(meta.z);
    const TravRay& r = q.r;
    if (counts != nullptr) {
        counts->boxes += static_cast<unsigned>(present);
        countReferenceBoxes(__ldg(np), __ldg(np + 1), __ldg(np + 2), __ldg(np + 3), __ldg(np + 4), __ldg(np + 5),
                            meta.w, r, q.tmin, q.tmax, *counts);
    }
    float e0 = 0.0f, e1 = 0.0f, e2 = 0.0f, e3 = 0.0f;
    unsigned mask;
    {
        // Near and far planes per axis by the sign of the inverse direction:
        // axis a's lo array is np[2a], its hi array np[2a + 1].
        const unsigned sx = r.planes & 1u;
        const unsigned sy = (r.planes >> 1) & 1u;
        const unsigned sz = (r.planes >> 2) & 1u;
        const float4 nx = __ldg(np + sx);
        const float4 fx = __ldg(np + (1u - sx));
        const float4 ny = __ldg(np + 2u + sy);
        const float4 fy = __ldg(np + (3u - sy));
        const float4 nz = __ldg(np + 4u + sz);
        const float4 fz = __ldg(np + (5u - sz));
        mask = (slabTestOrdered(nx.x, fx.x, ny.x, fy.x, nz.x, fz.x, r, q.tmin, q.tmax, e0) ? 1u : 0u) |
               (slabTestOrdered(nx.y, fx.y, ny.y, fy.y, nz.y, fz.y, r, q.tmin, q.tmax, e1) ? 2u : 0u) |
               (slabTestOrdered(nx.z, fx.z, ny.z, fy.z, nz.z, fz.z, r, q.tmin, q.tmax, e2) ? 4u : 0u) |
               (slabTestOrdered(nx.w, fx.w, ny.w, fy.w, nz.w, fz.w, r, q.tmin, q.tmax, e3) ? 8u : 0u);
        // Absent children (zero boxes) are tested too and masked off here.
        mask &= (1u << present) - 1u;
    }
    if (mask == 0u) {
        return kStepPop;
    }
    int remaining = __popc(mask);
    if (q.sp + remaining - 1 > stack_size) {
        atomicOr(error_flag, 1u);
        return kStepFinished;
    }
    const unsigned packed = (r.neg < 4u ? (meta.x >> (8u * r.neg)) : (meta.y >> (8u * (r.neg - 4u)))) & 0xFFu;
#pragma unroll
    for (int position = 3; position >= 0; --position) {
        if (position >= present) {
            continue;
        }
        const unsigned c = (packed >> (2 * position)) & 3u;
        if (((mask >> c) & 1u) == 0u) {
            continue;
        }
        const std::uint32_t child = c == 0u ? ch.x : (c == 1u ? ch.y : (c == 2u ? ch.z : ch.w));
        if (--remaining == 0) {
            q.ref = child;
        } else {
            const float entry = c == 0u ? e0 : (c == 1u ? e1 : (c == 2u ? e2 : e3));
            pushEntry(stack + q.sp * stride, child, entry);
            ++q.sp;
        }
    }
    return kStepDescend;
}

// A leaf. In the TLAS: spheres, scene triangles and instances in leaf order; an
// instance is entered at once (the rest of the leaf and an exit marker are
// pushed). In a BLAS: the current instance's triangles.
template <typename Stack>
__device__ __forceinline__ int leafStep(const DevScene& s, TraceState& q, const SkipRule& skip, Stack* stack,
                                        int stride, int stack_size, unsigned int* error_flag,
                                        TraversalCounts* counts, bool any)
{
    const std::uint32_t first = q.ref & kLeafFirstMask;
    const std::uint32_t count = ((q.ref >> 28) & 7u) + 1u;
    const bool in_mesh = q.inst_pos != kNoPrim;
    // One loop and one triangle test serve TLAS leaves (spheres, scene
    // triangles, instances) and mesh leaves (the current instance's triangles),
    // which keeps the traversal's code small.
    for (std::uint32_t k = 0; k < count; ++k) {
        const std::uint32_t pos = first + k;
        int kind = kObjTriangle;
        std::uint32_t index = pos;
        int mode = kSphereTestBoth;
        if (!in_mesh) {
            const DevObject obj = s.objects[pos];
            if (pos == skip.light_object_pos) {
                continue;
            }
            if (obj.kind == kObjInstance) {
                if (q.sp + 2 > stack_size) {
                    atomicOr(error_flag, 1u);
                    return kStepFinished;
                }
                if (k + 1 < count) {
                    pushEntry(stack + q.sp * stride, leafRef(pos + 1, count - k - 1), -INFINITY);
                    ++q.sp;
                }
                pushEntry(stack + q.sp * stride, kExitMarker, 0.0f);
                ++q.sp;
                const DevInstance& inst = s.instances[obj.index];
                if (counts != nullptr) {
                    counts->instances += 1;
                    counts->reference_boxes += 1; // the BLAS root
                }
                q.changeSpace(affinePoint(inst.to_object, q.origin), affineVector(inst.to_object, q.dir));
                q.inst_pos = pos;
                q.ref = inst.root;
                return kStepDescend;
            }
            kind = static_cast<int>(obj.kind);
            index = obj.index;
            if (pos == skip.object_pos) {
                if (kind == kObjTriangle || skip.sphere_mode == kSphereSkipAll) {
                    continue;
                }
                mode = skip.sphere_mode;
            }
        } else if (pos == skip.tri_pos && q.inst_pos == skip.object_pos) {
            continue;
        }
        float t;
        float b0 = 0.0f, b1 = 0.0f, b2 = 0.0f;
        bool h;
        if (kind == kObjTriangle) {
            const float4* tp = reinterpret_cast<const float4*>(s.triangles + index);
            if (counts != nullptr && (!in_mesh || q.r.usable)) {
                counts->triangles += 1;
            }
            h = q.r.usable &&
                intersectTriangle(q.r, __ldg(tp), __ldg(tp + 1), __ldg(tp + 2), q.tmin, q.tmax, t, b0, b1, b2);
        } else {
            if (counts != nullptr) {
                counts->spheres += 1;
            }
            h = intersectSphere(q.r, q.dir, s.spheres[index], kind == kObjSphereWide, q.tmin, q.tmax, mode, t);
        }
        if (h) {
            q.found = true;
            q.tmax = t;
            q.hit = {t, in_mesh ? q.inst_pos : pos, kind == kObjTriangle ? index : kNoPrim, b0, b1, b2};
            if (any) {
                return kStepFinished;
            }
        }
    }
    return kStepPop;
}

// Pops the next entry still worth visiting into `ref`; false when none is left.
// An exit marker returns the ray to world space; an entry whose box is entered
// beyond the current hit is dropped (accel/bvh.hpp:240-247).
__device__ __forceinline__ bool popNext(TraceState& q, const uint2* stack, int stride)
{
    for (;;) {
        if (q.sp == 0) {
            return false;
        }
        --q.sp;
        const uint2 e = stack[q.sp * stride];
        if (e.x == kExitMarker) {
            q.changeSpace(q.origin, q.dir);
            q.inst_pos = kNoPrim;
            continue;
        }
        if (__uint_as_float(e.y) > q.tmax) {
            continue;
        }
        q.ref = e.x;
        return true;
    }
}

// The same for 4-byte entries: no entry distance, so nothing is dropped here;
// the popped node's or leaf's own tests cull it.
__device__ __forceinline__ bool popNext(TraceState& q, const unsigned* stack, int stride)
{
    for (;;) {
        if (q.sp == 0) {
            return false;
        }
        --q.sp;
        const unsigned ref = stack[q.sp * stride];
        if (ref == kExitMarker) {
            q.changeSpace(q.origin, q.dir);
            q.inst_pos = kNoPrim;
            continue;
        }
        q.ref = ref;
        return true;
    }
}

// One turn of a query in a persistent kernel; returns whether the query has more
// work (false: finished). LOOP picks how much a turn does (the wavefront's
// autotuner chooses per workload; both visit the same nodes and leaves in the
// same order):
//   kLoopNodesThenLeaf  descend through interior nodes, then handle the leaf
//                       reached, so the lanes of a warp move through each phase
//                       together;
//   kLoopOneStep        one node or one leaf, so lanes return to take new rays
//                       sooner;
//   kLoopQuery          the whole query in one turn, through the out-of-line
//                       traversal (a function of its own: the calling kernel's
//                       state is saved around the call, and the traversal loop
//                       has the registers to itself).
enum TraceLoop : int { kLoopNodesThenLeaf = 0, kLoopOneStep = 1, kLoopQuery = 2 };

template <bool COUNT, bool HOLD, typename Stack>
static __device__ __noinline__ bool traceSceneOutOfLine(const DevScene& s, float3 origin, float3 dir, float tmin,
                                                        float& tmax, const SkipRule& skip, TraceHit& hit,
                                                        Stack* stack, int stride, int stack_size,
                                                        unsigned int* error_flag, TraversalCounts* counts, bool any);

template <int LOOP, typename Stack>
__device__ __forceinline__ bool traceAdvance(const DevScene& s, TraceState& q, const SkipRule& skip, Stack* stack,
                                             int stride, int stack_size, unsigned int* error_flag,
                                             TraversalCounts* counts, bool any)
{
    if constexpr (LOOP == kLoopQuery) {
        float tmax = q.tmax;
        TraceHit hit;
        q.found = traceSceneOutOfLine<false, false>(s, q.origin, q.dir, q.tmin, tmax, skip, hit, stack, stride,
                                                    stack_size, error_flag, nullptr, any);
        if (q.found) {
            q.tmax = tmax;
            q.hit = hit;
        }
        return false;
    }
    q.settle();
    int step = kStepDescend;
    if constexpr (LOOP == kLoopOneStep) {
        step = (q.ref & kLeafBit) == 0u ? nodeStep(s.nodes, q, stack, stride, stack_size, error_flag, counts)
                                        : leafStep(s, q, skip, stack, stride, stack_size, error_flag, counts, any);
    } else {
        while (step == kStepDescend && (q.ref & kLeafBit) == 0u) {
            step = nodeStep(s.nodes, q, stack, stride, stack_size, error_flag, counts);
        }
        if (step == kStepDescend) {
            step = leafStep(s, q, skip, stack, stride, stack_size, error_flag, counts, any);
        }
    }
    if (step == kStepFinished) {
        return false;
    }
    return step == kStepDescend || popNext(q, stack, stride);
}

// Traverses the scene for the nearest hit in (tmin, tmax) (any = false), or for
// any hit (any = true). On return `tmax` is the nearest hit distance. The stack
// overflow bound (TLAS depth + BLAS depth + 2) is checked on the host before
// launch, so pushes never exceed `stack_size`. It takes one step (a node or a
// leaf) per loop turn: inside the megakernel, the nested node/leaf loops of
// traceAdvance measured 3.4x slower.
//
// HOLD keeps the node table's address in registers for the whole query. Read
// through `s` at every node step instead, it comes from wherever the caller
// keeps the scene (local memory, for a caller of the out-of-line copy) and is
// reloaded after every stack push, a store the compiler cannot tell apart from
// it: one more dependent load in front of every node fetch. Holding it measured
// 2.7% faster in the megakernel (128 registers a thread) and 3-4% slower in the
// wavefront's persistent kernels, whose 96-register budget then spills.
template <bool HOLD, typename Stack>
__device__ __forceinline__ bool traceSceneBody(const DevScene& s, float3 origin, float3 dir, float tmin, float& tmax,
                                               const SkipRule& skip, TraceHit& hit, Stack* stack, int stride,
                                               int stack_size, unsigned int* error_flag, TraversalCounts* counts,
                                               bool any)
{
    if (counts != nullptr) {
        counts->rays += 1;
    }
    TraceState q;
    if (!traceBegin(s, q, origin, dir, tmin, tmax)) {
        return false;
    }
    if (counts != nullptr) {
        counts->reference_boxes += 1; // the TLAS root
    }
    const DevNode* const held_nodes = s.nodes;
    for (;;) {
        q.settle();
        const int step = (q.ref & kLeafBit) == 0u
                             ? nodeStep(HOLD ? held_nodes : s.nodes, q, stack, stride, stack_size, error_flag, counts)
                             : leafStep(s, q, skip, stack, stride, stack_size, error_flag, counts, any);
        if (step == kStepFinished || (step == kStepPop && !popNext(q, stack, stride))) {
            break;
        }
    }
    if (q.found) {
        tmax = q.tmax;
        hit = q.hit;
    }
    return q.found;
}

// One out-of-line copy serving closest-hit and any-hit queries alike, which
// keeps the kernels that call it small enough for the instruction cache. COUNT
// selects the copy that counts work (the counting kernels); the timed kernels'
// copy has no counting code at all.
template <bool COUNT, bool HOLD, typename Stack>
static __device__ __noinline__ bool traceSceneOutOfLine(const DevScene& s, float3 origin, float3 dir, float tmin,
                                                        float& tmax, const SkipRule& skip, TraceHit& hit,
                                                        Stack* stack, int stride, int stack_size,
                                                        unsigned int* error_flag, TraversalCounts* counts, bool any)
{
    return traceSceneBody<HOLD>(s, origin, dir, tmin, tmax, skip, hit, stack, stride, stack_size, error_flag,
                                COUNT ? counts : nullptr, any);
}

// A query from a caller that keeps its state across the call (the megakernel),
// closest hit or any hit as `any` says. INLINE places the traversal in the
// caller instead of calling the shared copy: no call, no registers saved around
// it, but a larger kernel. Which is faster depends on the scene (the
// megakernel's autotuner picks). COUNT adds the work counts into `counts`;
// without it `counts` is ignored.
template <bool INLINE = false, bool COUNT = false, typename Stack>
ALB_DEV bool traceQuery(const DevScene& s, float3 origin, float3 dir, float tmin, float& tmax, const SkipRule& skip,
                        TraceHit& hit, Stack* stack, int stride, int stack_size, unsigned int* error_flag,
                        TraversalCounts* counts, bool any)
{
    if constexpr (INLINE) {
        return traceSceneBody<true>(s, origin, dir, tmin, tmax, skip, hit, stack, stride, stack_size, error_flag,
                                    COUNT ? counts : nullptr, any);
    } else {
        return traceSceneOutOfLine<COUNT, true>(s, origin, dir, tmin, tmax, skip, hit, stack, stride, stack_size,
                                                error_flag, counts, any);
    }
}

template <bool ANY, bool INLINE = false, bool COUNT = false, typename Stack>
ALB_DEV bool traceScene(const DevScene& s, float3 origin, float3 dir, float tmin, float& tmax, const SkipRule& skip,
                        TraceHit& hit, Stack* stack, int stride, int stack_size, unsigned int* error_flag,
                        TraversalCounts* counts = nullptr)
{
    return traceQuery<INLINE, COUNT>(s, origin, dir, tmin, tmax, skip, hit, stack, stride, stack_size, error_flag,
                                     counts, ANY);
}

} // namespace albedo_b200
