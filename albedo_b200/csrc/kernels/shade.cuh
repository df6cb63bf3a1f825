// Surface shading in FP32: hit resolution, textures, materials, BSDF lobes,
// lights and next-event estimation pieces.
//
// Each function restates the reference function cited beside it, in the same
// order of operations, so that FP32 results follow the FP64 reference to
// rounding; branch decisions on random numbers differ only on a set of measure
// about 2^-24 per decision.
#pragma once

#include "traverse.cuh"

namespace albedo_b200 {

// ------------------------------------------------------------------ hit resolution

// A surface point as HitRecord holds it (scene/hit_record.hpp:13-33), with the
// normals facing the incoming ray, plus what shading needs to find its material.
struct Surface {
    float3 p;
    float3 n;   // geometric, facing the ray
    float3 ns;  // shading, flipped with n
    float3 sphere_outward; // unit outward normal of a sphere hit (texture coordinates)
    bool front;
    bool is_sphere;
    float b0, b1, b2;
    std::uint32_t tri_pos;
    std::uint32_t obj_pos;
    std::uint32_t object_id;
    std::uint32_t material;
};

// Smooth-shading normal from the corner normals and the barycentric weights of
// `p` recomputed from the point (geometry/mesh_geometry.cpp:53-64 with
// geometry/triangle.cpp:182-195). Falls back to the face normal when the blend
// nearly cancels.
ALB_DEV float3 blendedNormal(const DevTriangle& tri, const DevTriangleAttr& at, float3 p)
{
    const float3 v0 = mk(tri.v0x, tri.v0y, tri.v0z);
    const float3 e1 = mk(tri.v1x, tri.v1y, tri.v1z) - v0;
    const float3 e2 = mk(tri.v2x, tri.v2y, tri.v2z) - v0;
    const float3 off = p - v0;
    const float3 an = cross(e1, e2);
    const float area2 = lengthSquared(an);
    const float b1 = dot(cross(off, e2), an) / area2;
    const float b2 = dot(cross(e1, off), an) / area2;
    const float b0 = 1.0f - b1 - b2;
    const float3 blended = mk(at.cn0x, at.cn0y, at.cn0z) * b0 + mk(at.cn1x, at.cn1y, at.cn1z) * b1 +
                           mk(at.cn2x, at.cn2y, at.cn2z) * b2;
    if (!(lengthSquared(blended) >= 1e-12f)) {
        return mk(at.nx, at.ny, at.nz);
    }
    return normalized(blended);
}

// The reported hit's distance recomputed once in FP64 (traversal decided which
// primitive is nearest in FP32): the sphere root closest to the FP32 one, or the
// watertight triangle distance, with instance rays taken to object space in FP64.
ALB_DEV double refinedDistance(const DevScene& s, float3 origin, float3 dir, const TraceHit& h)
{
    const DevObject obj = s.objects[h.obj_pos];
    const double ox = origin.x, oy = origin.y, oz = origin.z;
    const double dx = dir.x, dy = dir.y, dz = dir.z;
    if (obj.kind == kObjSphere || obj.kind == kObjSphereWide) {
        const DevSphere sp = s.spheres[obj.index];
        const double cx = ox - sp.cx, cy = oy - sp.cy, cz = oz - sp.cz;
        const double a = dx * dx + dy * dy + dz * dz;
        const double hh = dx * cx + dy * cy + dz * cz;
        const double r2 = static_cast<double>(sp.r) * sp.r;
        const double c = (cx * cx + cy * cy + cz * cz) - r2;
        const double k = hh / a;
        const double lx = cx - dx * k, ly = cy - dy * k, lz = cz - dz * k;
        const double disc = fmax(a * (r2 - (lx * lx + ly * ly + lz * lz)), 0.0);
        const double q = -(hh + copysign(sqrt(disc), hh));
        if (q == 0.0) {
            return 0.0;
        }
        const double r0 = q / a;
        const double r1 = c / q;
        return fabs(r0 - h.t) < fabs(r1 - h.t) ? r0 : r1;
    }
    double px = ox, py = oy, pz = oz, qx = dx, qy = dy, qz = dz;
    if (obj.kind == kObjInstance) {
        const double* m = s.instance_to_object64 + 12 * obj.index;
        px = m[0] * ox + m[1] * oy + m[2] * oz + m[3];
        py = m[4] * ox + m[5] * oy + m[6] * oz + m[7];
        pz = m[8] * ox + m[9] * oy + m[10] * oz + m[11];
        qx = m[0] * dx + m[1] * dy + m[2] * dz;
        qy = m[4] * dx + m[5] * dy + m[6] * dz;
        qz = m[8] * dx + m[9] * dy + m[10] * dz;
    }
    const DevTriangle tri = s.triangles[h.tri_pos];
    const double mx = fabs(qx), my = fabs(qy), mz = fabs(qz);
    const int kz = mx > my ? (mx > mz ? 0 : 2) : (my > mz ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    const double q3[3] = {qx, qy, qz};
    if (q3[kz] < 0.0) {
        const int t = kx;
        kx = ky;
        ky = t;
    }
    const double sx = q3[kx] / q3[kz], sy = q3[ky] / q3[kz], sz = 1.0 / q3[kz];
    const double A[3] = {tri.v0x - px, tri.v0y - py, tri.v0z - pz};
    const double B[3] = {tri.v1x - px, tri.v1y - py, tri.v1z - pz};
    const double C[3] = {tri.v2x - px, tri.v2y - py, tri.v2z - pz};
    const double ax = A[kx] - sx * A[kz], ay = A[ky] - sy * A[kz];
    const double bx = B[kx] - sx * B[kz], by = B[ky] - sy * B[kz];
    const double cx = C[kx] - sx * C[kz], cy = C[ky] - sy * C[kz];
    const double u = cx * by - cy * bx;
    const double v = ax * cy - ay * cx;
    const double w = bx * ay - by * ax;
    const double det = u + v + w;
    if (det == 0.0) {
        return h.t;
    }
    return (u * (sz * A[kz]) + v * (sz * B[kz]) + w * (sz * C[kz])) / det;
}

// Scene::intersect's record (scene/scene.cpp:107-133) for a TraceHit.
ALB_DEV void resolveHit(const DevScene& s, float3 origin, float3 dir, const TraceHit& h, Surface& out)
{
    const DevObject obj = s.objects[h.obj_pos];
    out.obj_pos = h.obj_pos;
    out.object_id = obj.id;
    out.material = obj.material;
    out.tri_pos = h.tri_pos;
    out.b0 = h.b0;
    out.b1 = h.b1;
    out.b2 = h.b2;
    float3 n;
    float3 ns;
    if (obj.kind == kObjSphere || obj.kind == kObjSphereWide) {
        const DevSphere sp = s.spheres[obj.index];
        // The hit point from the FP64 distance: FP32 o + t d loses the walls' 1e4-scale digits.
        const double t = refinedDistance(s, origin, dir, h);
        out.p = mk(static_cast<float>(origin.x + dir.x * t), static_cast<float>(origin.y + dir.y * t),
                   static_cast<float>(origin.z + dir.z * t));
        n = normalized(mk(static_cast<float>(origin.x + dir.x * t - sp.cx),
                          static_cast<float>(origin.y + dir.y * t - sp.cy),
                          static_cast<float>(origin.z + dir.z * t - sp.cz)));
        ns = n;
        out.sphere_outward = n;
        out.is_sphere = true;
    } else {
        out.is_sphere = false;
        const DevTriangle tri = s.triangles[h.tri_pos];
        const DevTriangleAttr at = s.attrs[h.tri_pos];
        const float3 v0 = mk(tri.v0x, tri.v0y, tri.v0z);
        const float3 p_local = v0 + (mk(tri.v1x, tri.v1y, tri.v1z) - v0) * h.b1 + (mk(tri.v2x, tri.v2y, tri.v2z) - v0) * h.b2;
        const float3 face = mk(at.nx, at.ny, at.nz);
        if (obj.kind == kObjTriangle) {
            out.p = p_local;
            n = face;
            ns = face;
        } else {
            // MeshInstance::intersect and worldShadingNormal (geometry/mesh_instance.cpp:32-60).
            const DevInstance& inst = s.instances[obj.index];
            out.p = affinePoint(inst.to_world, p_local);
            const float3 wn = affineTransposedVector(inst.to_object, face);
            n = normalized(wn);
            ns = n;
            if (at.smooth != 0.0f) {
                const float3 local_ns = blendedNormal(tri, at, p_local);
                if (!(local_ns.x == face.x && local_ns.y == face.y && local_ns.z == face.z)) {
                    const float3 wsn = affineTransposedVector(inst.to_object, local_ns);
                    ns = isNormalF(lengthSquared(wsn)) ? normalized(wsn) : n;
                }
            }
        }
    }
    out.front = dot(dir, n) < 0.0f;
    out.n = out.front ? n : -n;
    out.ns = out.front ? ns : -ns;
}

// Texture coordinates of a hit (geometry/sphere.cpp:137-148, geometry/triangle.cpp:166-174).
ALB_DEV float2 surfaceUv(const DevScene& s, const Surface& sf)
{
    if (sf.is_sphere) {
        const float3 n = sf.sphere_outward;
        const float longitude = atan2f(-n.z, n.x) + kPiF;
        const float latitude = acosf(fminf(fmaxf(-n.y, -1.0f), 1.0f));
        return make_float2(longitude / (2.0f * kPiF), latitude / kPiF);
    }
    const DevTriangleAttr at = s.attrs[sf.tri_pos];
    return make_float2(sf.b0 * at.u0 + sf.b1 * at.u1 + sf.b2 * at.u2, sf.b0 * at.v0 + sf.b1 * at.v1 + sf.b2 * at.v2);
}

// ------------------------------------------------------------------ Perlin noise

// Perlin's published permutation of 0..255 ("Improving Noise", SIGGRAPH 2002),
// which texture/perlin_noise.cpp:17-36 uses so patterns match the published code.
__constant__ unsigned char c_perm[256] = {
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

ALB_DEV unsigned hashed(unsigned i) { return c_perm[i & 255u]; }

// cellPosition (texture/perlin_noise.cpp:74-86): cell index wrapped to 256, offset in [0, 1).
ALB_DEV unsigned cellOf(float coordinate, float& offset)
{
    const float f = floorf(coordinate);
    float wrapped = fmodf(f, 256.0f);
    if (wrapped < 0.0f) {
        wrapped += 256.0f;
    }
    offset = coordinate - f;
    return static_cast<unsigned>(wrapped);
}

ALB_DEV float fade(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }
ALB_DEV float lerpf(float t, float a, float b) { return a + t * (b - a); }

// gradient (texture/perlin_noise.cpp:99-110).
ALB_DEV float grad(unsigned hash, float x, float y, float z)
{
    const unsigned h = hash & 15u;
    const float u = h < 8u ? x : y;
    float v = z;
    if (h < 4u) {
        v = y;
    } else if (h == 12u || h == 14u) {
        v = x;
    }
    return ((h & 1u) == 0u ? u : -u) + ((h & 2u) == 0u ? v : -v);
}

// perlinNoise (texture/perlin_noise.cpp:114-138).
static __device__ __noinline__ float perlinNoise(float3 p)
{
    if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z)) {
        return 0.0f;
    }
    float x, y, z;
    const unsigned xi = cellOf(p.x, x);
    const unsigned yi = cellOf(p.y, y);
    const unsigned zi = cellOf(p.z, z);
    const float u = fade(x);
    const float v = fade(y);
    const float w = fade(z);
    const unsigned a = hashed(xi) + yi;
    const unsigned aa = hashed(a) + zi;
    const unsigned ab = hashed(a + 1u) + zi;
    const unsigned b = hashed(xi + 1u) + yi;
    const unsigned ba = hashed(b) + zi;
    const unsigned bb = hashed(b + 1u) + zi;
    return lerpf(w,
                 lerpf(v, lerpf(u, grad(hashed(aa), x, y, z), grad(hashed(ba), x - 1.0f, y, z)),
                       lerpf(u, grad(hashed(ab), x, y - 1.0f, z), grad(hashed(bb), x - 1.0f, y - 1.0f, z))),
                 lerpf(v, lerpf(u, grad(hashed(aa + 1u), x, y, z - 1.0f), grad(hashed(ba + 1u), x - 1.0f, y, z - 1.0f)),
                       lerpf(u, grad(hashed(ab + 1u), x, y - 1.0f, z - 1.0f),
                             grad(hashed(bb + 1u), x - 1.0f, y - 1.0f, z - 1.0f))));
}

// turbulence, 7 octaves (texture/perlin_noise.cpp:140-150).
ALB_DEV float turbulence(float3 p)
{
    float sum = 0.0f;
    float weight = 1.0f;
    for (int octave = 0; octave < 7; ++octave) {
        sum += weight * fabsf(perlinNoise(p));
        weight *= 0.5f;
        p = mk(p.x * 2.0f, p.y * 2.0f, p.z * 2.0f);
    }
    return sum;
}

// PerlinPattern::weightAt (texture/perlin_pattern.cpp:11-23).
ALB_DEV float patternWeight(float scale, float veins, float3 point)
{
    const float3 scaled = mk(point.x * scale, point.y * scale, point.z * scale);
    const float swirl = turbulence(scaled);
    if (veins == 0.0f) {
        return fminf(swirl, 1.0f);
    }
    const float weight = (1.0f + sinf(scaled.x + veins * swirl)) / 2.0f;
    return isnan(weight) ? 0.5f : weight;
}

// ------------------------------------------------------------------ GGX and Fresnel

// GgxDistribution (scattering/ggx_distribution.cpp:28-111).
struct Ggx {
    float alpha;
    ALB_DEV float density(float3 m) const
    {
        if (m.z <= 0.0f) {
            return 0.0f;
        }
        const float a2 = alpha * alpha;
        const float den = m.z * m.z * (a2 - 1.0f) + 1.0f;
        return a2 / (kPiF * den * den);
    }
    ALB_DEV float lambda(float3 w) const
    {
        const float cos2 = w.z * w.z;
        if (cos2 == 0.0f) {
            return INFINITY;
        }
        const float tan2 = (w.x * w.x + w.y * w.y) / cos2;
        return (sqrtf(1.0f + alpha * alpha * tan2) - 1.0f) / 2.0f;
    }
    ALB_DEV float masking(float3 w) const { return 1.0f / (1.0f + lambda(w)); }
    ALB_DEV float maskingShadowing(float3 wo, float3 wi) const { return 1.0f / (1.0f + lambda(wo) + lambda(wi)); }
    ALB_DEV float3 sampleVisibleNormal(float3 wo, float ux, float uy) const
    {
        const float3 view = normalized(mk(alpha * wo.x, alpha * wo.y, wo.z));
        const float len2 = view.x * view.x + view.y * view.y;
        const float3 first = len2 > 0.0f ? mk(-view.y, view.x, 0.0f) / sqrtf(len2) : mk(1.0f, 0.0f, 0.0f);
        const float3 second = cross(view, first);
        const float radius = sqrtf(ux);
        const float phi = 2.0f * kPiF * uy;
        float sp, cp;
        sincosf(phi, &sp, &cp);
        const float t1 = radius * cp;
        const float blend = (1.0f + view.z) / 2.0f;
        const float t2 = (1.0f - blend) * sqrtf(fmaxf(0.0f, 1.0f - t1 * t1)) + blend * radius * sp;
        const float lift = sqrtf(fmaxf(0.0f, 1.0f - t1 * t1 - t2 * t2));
        const float3 hn = first * t1 + second * t2 + view * lift;
        return normalized(mk(alpha * hn.x, alpha * hn.y, fmaxf(0.0f, hn.z)));
    }
    ALB_DEV float visibleNormalPdf(float3 wo, float3 m) const
    {
        const float facing = dot(wo, m);
        if (wo.z <= 0.0f || facing <= 0.0f) {
            return 0.0f;
        }
        return masking(wo) * facing * density(m) / wo.z;
    }
};

// Unpolarized reflectance at a smooth boundary with a real relative index
// (scattering/fresnel.cpp:17-47; the complex form with zero imaginary part).
ALB_DEV float fresnelDielectric(float cos_i, float eta)
{
    if (cos_i < 0.0f) {
        cos_i = -cos_i;
        eta = 1.0f / eta;
    }
    cos_i = fminf(cos_i, 1.0f);
    if (eta == 1.0f) {
        return 0.0f;
    }
    const float sin2_i = 1.0f - cos_i * cos_i;
    const float sin2_t = sin2_i / (eta * eta);
    if (sin2_t >= 1.0f) {
        return 1.0f;
    }
    const float cos_t = sqrtf(1.0f - sin2_i / (eta * eta));
    const float rp = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    const float rs = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    return (rp * rp + rs * rs) / 2.0f;
}

// Complex arithmetic for the conductor Fresnel equations (std::complex semantics,
// principal square root with non-negative real part).
struct Cpx {
    float re, im;
};
ALB_DEV Cpx cmul(Cpx a, Cpx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
ALB_DEV Cpx cdiv(Cpx a, Cpx b)
{
    const float den = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / den, (a.im * b.re - a.re * b.im) / den};
}
ALB_DEV Cpx csqrt(Cpx z)
{
    if (z.re == 0.0f && z.im == 0.0f) {
        return {0.0f, z.im};
    }
    const float r = hypotf(z.re, z.im);
    if (z.re >= 0.0f) {
        const float t = sqrtf(0.5f * (r + z.re));
        return {t, z.im / (2.0f * t)};
    }
    const float t = sqrtf(0.5f * (r - z.re));
    return {fabsf(z.im) / (2.0f * t), copysignf(t, z.im)};
}

// reflectance() of scattering/fresnel.cpp:17-25 for eta + i k.
static __device__ __noinline__ float conductorReflectance(float cos_i, float eta, float k)
{
    const Cpx e{eta, k};
    const float sin2 = 1.0f - cos_i * cos_i;
    const Cpx e2 = cmul(e, e);
    const Cpx ratio = cdiv(Cpx{sin2, 0.0f}, e2);
    const Cpx cos_t = csqrt(Cpx{1.0f - ratio.re, -ratio.im});
    const Cpx ec = {e.re * cos_i, e.im * cos_i};
    const Cpx rp = cdiv(Cpx{ec.re - cos_t.re, ec.im - cos_t.im}, Cpx{ec.re + cos_t.re, ec.im + cos_t.im});
    const Cpx ect = cmul(e, cos_t);
    const Cpx rs = cdiv(Cpx{cos_i - ect.re, -ect.im}, Cpx{cos_i + ect.re, ect.im});
    return ((rp.re * rp.re + rp.im * rp.im) + (rs.re * rs.re + rs.im * rs.im)) / 2.0f;
}

// fresnelConductor (scattering/fresnel.cpp:49-58).
ALB_DEV float3 fresnelConductor(float cos_i, float3 eta, float3 k)
{
    cos_i = fminf(fmaxf(cos_i, 0.0f), 1.0f);
    return mk(conductorReflectance(cos_i, eta.x, k.x), conductorReflectance(cos_i, eta.y, k.y),
              conductorReflectance(cos_i, eta.z, k.z));
}

ALB_DEV float3 reflectAbout(float3 w, float3 n) { return n * (2.0f * dot(w, n)) - w; }

// refract (scattering/specular.cpp:9-22); false under total internal reflection.
ALB_DEV bool refractThrough(float3 w, float3 n, float eta, float3& out)
{
    const float cos_i = dot(w, n);
    const float sin2_t = fmaxf(0.0f, 1.0f - cos_i * cos_i) / (eta * eta);
    if (sin2_t >= 1.0f) {
        return false;
    }
    const float cos_t = sqrtf(1.0f - sin2_t);
    out = -w / eta + n * (cos_i / eta - cos_t);
    return true;
}

// ------------------------------------------------------------------ lobes (local space)

struct ScatterSample {
    float3 dir;
    float3 weight;
    float pdf;
    bool specular;
};

enum LobeKind : int { kLobeLambert = 0, kLobeConductor = 1, kLobeDielectric = 2 };

struct Lobe {
    int kind;
    float3 c0;  // Lambert albedo; conductor eta
    float3 c1;  // conductor k
    float alpha;
    float eta;  // dielectric relative index
};

constexpr float kSmoothAlpha = 1e-4f;

ALB_DEV float3 gray(float v) { return mk(v, v, v); }

ALB_DEV bool dielectricSmooth(const Lobe& l) { return l.alpha < kSmoothAlpha || l.eta == 1.0f; }

// refractionHalfVector (scattering/dielectric_lobe.cpp:30-46).
ALB_DEV bool refractionHalfVector(float3 wo, float3 wi, float eta, float3& m)
{
    const float3 sum = wo + wi * eta;
    if (lengthSquared(sum) == 0.0f) {
        return false;
    }
    m = normalized(sum);
    if (m.z < 0.0f) {
        m = -m;
    }
    return !(dot(wo, m) <= 0.0f || dot(wi, m) >= 0.0f);
}

ALB_DEV float refractionDenominator(float3 wo, float3 wi, float3 m, float eta)
{
    const float d = eta * dot(wi, m) + dot(wo, m);
    return d * d;
}

// Lobe pdf (lambert_lobe.cpp:38-41, conductor_lobe.cpp:58-73, dielectric_lobe.cpp:159-186).
ALB_DEV float lobePdf(const Lobe& l, float3 wo, float3 wi)
{
    if (l.kind == kLobeLambert) {
        return wo.z > 0.0f ? (wi.z > 0.0f ? wi.z * kInvPiF : 0.0f) : 0.0f;
    }
    if (l.kind == kLobeConductor) {
        if (l.alpha < kSmoothAlpha || wo.z <= 0.0f || wi.z <= 0.0f) {
            return 0.0f;
        }
        const float3 m = normalized(wo + wi);
        const float facing = dot(wo, m);
        if (facing <= 0.0f) {
            return 0.0f;
        }
        return Ggx{l.alpha}.visibleNormalPdf(wo, m) / (4.0f * facing);
    }
    if (dielectricSmooth(l) || wo.z <= 0.0f || wi.z == 0.0f) {
        return 0.0f;
    }
    const Ggx ggx{l.alpha};
    if (wi.z > 0.0f) {
        const float3 m = normalized(wo + wi);
        const float facing = dot(wo, m);
        return ggx.visibleNormalPdf(wo, m) * fresnelDielectric(facing, l.eta) / (4.0f * facing);
    }
    float3 m;
    if (!refractionHalfVector(wo, wi, l.eta, m)) {
        return 0.0f;
    }
    const float jacobian = l.eta * l.eta * fabsf(dot(wi, m)) / refractionDenominator(wo, wi, m, l.eta);
    return ggx.visibleNormalPdf(wo, m) * (1.0f - fresnelDielectric(dot(wo, m), l.eta)) * jacobian;
}

// Lobe f(wo, wi) (lambert_lobe.cpp:17-20, conductor_lobe.cpp:18-32, dielectric_lobe.cpp:108-135).
ALB_DEV float3 lobeEvaluate(const Lobe& l, float3 wo, float3 wi)
{
    if (l.kind == kLobeLambert) {
        return (wo.z > 0.0f && wi.z > 0.0f) ? l.c0 * kInvPiF : gray(0.0f);
    }
    if (l.kind == kLobeConductor) {
        if (l.alpha < kSmoothAlpha || wo.z <= 0.0f || wi.z <= 0.0f) {
            return gray(0.0f);
        }
        const float3 m = normalized(wo + wi);
        const Ggx ggx{l.alpha};
        const float3 f = fresnelConductor(dot(wo, m), l.c0, l.c1);
        return f * (ggx.density(m) * ggx.maskingShadowing(wo, wi) / (4.0f * wo.z * wi.z));
    }
    if (dielectricSmooth(l) || wo.z <= 0.0f || wi.z == 0.0f) {
        return gray(0.0f);
    }
    const Ggx ggx{l.alpha};
    if (wi.z > 0.0f) {
        const float3 m = normalized(wo + wi);
        const float reflectance = fresnelDielectric(dot(wo, m), l.eta);
        return gray(reflectance * ggx.density(m) * ggx.maskingShadowing(wo, wi) / (4.0f * wo.z * wi.z));
    }
    float3 m;
    if (!refractionHalfVector(wo, wi, l.eta, m)) {
        return gray(0.0f);
    }
    const float transmittance = 1.0f - fresnelDielectric(dot(wo, m), l.eta);
    const float masking = ggx.masking(wo) * ggx.masking(wi);
    return gray(fabsf(dot(wi, m)) * dot(wo, m) * transmittance * ggx.density(m) * masking /
                (-wi.z * wo.z * refractionDenominator(wo, wi, m, l.eta)));
}

// Lobe sampling (lambert_lobe.cpp:22-36, conductor_lobe.cpp:34-56, dielectric_lobe.cpp:56-106, 137-157).
ALB_DEV bool lobeSample(const Lobe& l, float3 wo, float u_choice, float ux, float uy, ScatterSample& out)
{
    if (wo.z <= 0.0f) {
        return false;
    }
    if (l.kind == kLobeLambert) {
        const float3 wi = cosineHemisphere(ux, uy);
        if (wi.z <= 0.0f) {
            return false;
        }
        out = {wi, l.c0, wi.z * kInvPiF, false};
        return true;
    }
    if (l.kind == kLobeConductor) {
        if (l.alpha < kSmoothAlpha) {
            out = {reflectAbout(wo, mk(0.0f, 0.0f, 1.0f)), fresnelConductor(wo.z, l.c0, l.c1), 1.0f, true};
            return true;
        }
        const Ggx ggx{l.alpha};
        const float3 m = ggx.sampleVisibleNormal(wo, ux, uy);
        const float3 wi = reflectAbout(wo, m);
        const float pdf = lobePdf(l, wo, wi);
        if (wi.z <= 0.0f || pdf <= 0.0f) {
            return false;
        }
        const float3 f = fresnelConductor(dot(wo, m), l.c0, l.c1);
        out = {wi, f * (ggx.maskingShadowing(wo, wi) / ggx.masking(wo)), pdf, false};
        return true;
    }
    // Dielectric.
    if (dielectricSmooth(l)) {
        const float reflectance = fresnelDielectric(wo.z, l.eta);
        if (u_choice < reflectance) {
            out = {reflectAbout(wo, mk(0.0f, 0.0f, 1.0f)), gray(1.0f), reflectance, true};
            return true;
        }
        float3 wi;
        if (!refractThrough(wo, mk(0.0f, 0.0f, 1.0f), l.eta, wi)) {
            return false;
        }
        out = {wi, gray(1.0f / (l.eta * l.eta)), 1.0f - reflectance, true};
        return true;
    }
    const Ggx ggx{l.alpha};
    const float3 m = ggx.sampleVisibleNormal(wo, ux, uy);
    const float facing = dot(wo, m);
    if (facing <= 0.0f) {
        return false;
    }
    float3 wi;
    float3 weight;
    if (u_choice < fresnelDielectric(facing, l.eta)) {
        wi = reflectAbout(wo, m);
        if (wi.z <= 0.0f) {
            return false;
        }
        weight = gray(ggx.maskingShadowing(wo, wi) / ggx.masking(wo));
    } else {
        if (!refractThrough(wo, m, l.eta, wi) || wi.z >= 0.0f) {
            return false;
        }
        weight = gray(ggx.masking(wi) / (l.eta * l.eta));
    }
    const float pdf = lobePdf(l, wo, wi);
    if (pdf <= 0.0f) {
        return false;
    }
    out = {wi, weight, pdf, false};
    return true;
}

// ------------------------------------------------------------------ materials and scattering

// Scattering (scattering/scattering.cpp:10-54): a lobe in the shading frame with
// the geometric-side check.
struct Scattering {
    Lobe lobe;
    Onb basis;
    float3 geometric;

    ALB_DEV bool crossesSurface(float3 d) const
    {
        return (dot(d, basis.n) < 0.0f) != (dot(d, geometric) < 0.0f);
    }
    ALB_DEV float3 evaluate(float3 wo, float3 wi) const
    {
        if (crossesSurface(wo) || crossesSurface(wi)) {
            return gray(0.0f);
        }
        return lobeEvaluate(lobe, basis.toLocal(wo), basis.toLocal(wi));
    }
    ALB_DEV float pdf(float3 wo, float3 wi) const
    {
        if (crossesSurface(wo) || crossesSurface(wi)) {
            return 0.0f;
        }
        return lobePdf(lobe, basis.toLocal(wo), basis.toLocal(wi));
    }
    ALB_DEV bool sample(float3 wo, float u_choice, float ux, float uy, ScatterSample& out) const
    {
        if (crossesSurface(wo)) {
            return false;
        }
        if (!lobeSample(lobe, basis.toLocal(wo), u_choice, ux, uy, out)) {
            return false;
        }
        out.dir = basis.toWorld(out.dir);
        return !crossesSurface(out.dir);
    }
};

// Texture colour at a hit (constant, checker_texture.cpp:8-17, perlin_texture.cpp:7-11).
ALB_DEV float3 textureColor(const DevScene& s, const DevBasic& b, const Surface& sf)
{
    const float3 a = ld3(b.a);
    if (b.texture == kTexConstant) {
        return a;
    }
    if (b.texture == kTexChecker) {
        const float2 uv = surfaceUv(s, sf);
        const float sum = floorf(uv.x * b.s0) + floorf(uv.y * b.s0);
        return fabsf(fmodf(sum, 2.0f)) == 1.0f ? ld3(b.b) : a;
    }
    const float weight = patternWeight(b.s0, b.s1, sf.p);
    return a * (1.0f - weight) + ld3(b.b) * weight;
}

// Material -> Scattering (material/*.hpp, mix_material.cpp:7-11).
ALB_DEV Scattering scatteringAt(const DevScene& s, const Surface& sf)
{
    const DevMaterial& m = s.materials[sf.material];
    const DevBasic* b = &m.first;
    if (m.mix != 0u) {
        b = patternWeight(m.scale, m.veins, sf.p) < m.threshold ? &m.first : &m.second;
    }
    Scattering sc;
    sc.basis = Onb::fromNormal(sf.ns);
    sc.geometric = sf.n;
    if (b->kind == kDiffuse) {
        sc.lobe = {kLobeLambert, textureColor(s, *b, sf), gray(0.0f), 0.0f, 1.0f};
    } else if (b->kind == kConductor) {
        sc.lobe = {kLobeConductor, ld3(b->a), ld3(b->b), b->s0, 1.0f};
    } else {
        sc.lobe = {kLobeDielectric, gray(0.0f), gray(0.0f), b->s0, sf.front ? b->s1 : 1.0f / b->s1};
    }
    return sc;
}

// Material classes the wavefront renderer shades in separate kernels.
enum MaterialClass : int { kClassDiffuse = 0, kClassConductor = 1, kClassDielectric = 2, kClassMix = 3 };

ALB_DEV int materialClass(const DevScene& s, std::uint32_t obj_pos)
{
    const DevMaterial& m = s.materials[s.objects[obj_pos].material];
    return m.mix != 0u ? kClassMix : static_cast<int>(m.first.kind);
}

// scatteringAt for a material known to be of class CLASS, so that only that
// lobe's code is compiled into the kernel shading it.
template <int CLASS>
ALB_DEV Scattering scatteringAtClass(const DevScene& s, const Surface& sf)
{
    if constexpr (CLASS == kClassMix) {
        return scatteringAt(s, sf);
    } else {
        const DevBasic& b = s.materials[sf.material].first;
        Scattering sc;
        sc.basis = Onb::fromNormal(sf.ns);
        sc.geometric = sf.n;
        if constexpr (CLASS == kClassDiffuse) {
            sc.lobe = {kLobeLambert, textureColor(s, b, sf), gray(0.0f), 0.0f, 1.0f};
        } else if constexpr (CLASS == kClassConductor) {
            sc.lobe = {kLobeConductor, ld3(b.a), ld3(b.b), b.s0, 1.0f};
        } else {
            sc.lobe = {kLobeDielectric, gray(0.0f), gray(0.0f), b.s0, sf.front ? b.s1 : 1.0f / b.s1};
        }
        return sc;
    }
}

// ------------------------------------------------------------------ lights

struct LightSample {
    float3 dir;
    float3 radiance;
    float distance;
    float pdf;
    bool delta;
};

// coneTowards (light/area_light.cpp:31-53).
struct Cone {
    float3 axis;
    float distance;
    float tangent2;
    float cos_max;
    float one_minus_cos_max;
};

ALB_DEV bool coneTowards(const DevLight& l, float3 p, Cone& c)
{
    const float3 to_center = ld3(l.p) - p;
    const float d2 = lengthSquared(to_center);
    const float r2 = l.radius * l.radius;
    if (d2 <= r2) {
        return false;
    }
    const float d = sqrtf(d2);
    const float sin2_max = r2 / d2;
    const float cos_max = sqrtf(1.0f - sin2_max);
    const float omc = sin2_max / (1.0f + cos_max);
    if (!isNormalF(omc)) {
        return false;
    }
    c = {to_center / d, d, d2 - r2, cos_max, omc};
    return true;
}

ALB_DEV float3 skyRadiance(const DevLight& l, float3 dir)
{
    const float h = 0.5f * (dir.y + 1.0f);
    return ld3(l.e) * (1.0f - h) + ld3(l.z) * h;
}

// sampleIncidentLight (point_light.cpp:7-21, area_light.cpp:55-82, sky_light.cpp:15-24).
ALB_DEV bool sampleLight(const DevLight& l, float3 p, float ux, float uy, LightSample& out)
{
    if (l.kind == kLightPoint) {
        const float3 to = ld3(l.p) - p;
        const float d2 = lengthSquared(to);
        if (d2 == 0.0f) {
            return false;
        }
        const float d = sqrtf(d2);
        out = {to / d, ld3(l.e) / d2, d, 1.0f, true};
        return true;
    }
    if (l.kind == kLightArea) {
        Cone c;
        if (!coneTowards(l, p, c)) {
            return false;
        }
        const float omc = ux * c.one_minus_cos_max;
        const float cos_t = 1.0f - omc;
        const float sin2 = omc * (2.0f - omc);
        const float sin_t = sqrtf(sin2);
        const float phi = 2.0f * kPiF * uy;
        float sp, cp;
        sincosf(phi, &sp, &cp);
        const Onb basis = Onb::fromNormal(c.axis);
        const float3 dir = basis.toWorld(mk(sin_t * cp, sin_t * sp, cos_t));
        const float r2 = l.radius * l.radius;
        const float root = sqrtf(fmaxf(0.0f, r2 - c.distance * c.distance * sin2));
        out = {dir, ld3(l.e), c.tangent2 / (c.distance * cos_t + root), 1.0f / (2.0f * kPiF * c.one_minus_cos_max),
               false};
        return true;
    }
    const float3 dir = uniformSphere(ux, uy);
    out = {dir, skyRadiance(l, dir), INFINITY, uniformSpherePdf(), false};
    return true;
}

// incidentLightPdf (area_light.cpp:84-94; sky 1/4pi; point 0).
ALB_DEV float lightPdf(const DevLight& l, float3 p, float3 dir)
{
    if (l.kind == kLightPoint) {
        return 0.0f;
    }
    if (l.kind == kLightSky) {
        return uniformSpherePdf();
    }
    Cone c;
    if (!coneTowards(l, p, c)) {
        return 0.0f;
    }
    if (dot(dir, c.axis) < c.cos_max) {
        return 0.0f;
    }
    return 1.0f / (2.0f * kPiF * c.one_minus_cos_max);
}

// Veach's power heuristic (estimator/path_estimator.cpp:47-52).
ALB_DEV float powerHeuristic(float chosen, float other)
{
    const float c2 = chosen * chosen;
    const float total = c2 + other * other;
    return total > 0.0f ? c2 / total : 0.0f;
}

// shadowRange upper end (estimator/path_estimator.cpp:62-69).
ALB_DEV float shadowRangeMax(float distance)
{
    if (isinf(distance)) {
        return distance;
    }
    const float margin = fmaxf(distance * 1e-6f, 2.0f * 1e-7f);
    return distance - margin;
}

// Wachter & Binder, "A Fast and Robust Method for Avoiding Self-Intersection"
// (Ray Tracing Gems, ch. 6): moves `p` a few ulps along `n` in integer space, and
// by a fixed small distance near the origin where ulps vanish.
ALB_DEV float3 offsetOrigin(float3 p, float3 n)
{
    constexpr float kOrigin = 1.0f / 32.0f;
    constexpr float kFloatScale = 1.0f / 65536.0f;
    constexpr float kIntScale = 32.0f;
    const int ox = static_cast<int>(kIntScale * n.x);
    const int oy = static_cast<int>(kIntScale * n.y);
    const int oz = static_cast<int>(kIntScale * n.z);
    const float px = __int_as_float(__float_as_int(p.x) + (p.x < 0.0f ? -ox : ox));
    const float py = __int_as_float(__float_as_int(p.y) + (p.y < 0.0f ? -oy : oy));
    const float pz = __int_as_float(__float_as_int(p.z) + (p.z < 0.0f ? -oz : oz));
    return mk(fabsf(p.x) < kOrigin ? p.x + kFloatScale * n.x : px, fabsf(p.y) < kOrigin ? p.y + kFloatScale * n.y : py,
              fabsf(p.z) < kOrigin ? p.z + kFloatScale * n.z : pz);
}

// rayLeaving (estimator/surface_ray.hpp:26-31) with the FP32 skip rule.
ALB_DEV void rayLeaving(const Surface& sf, float3 dir, float3& origin, SkipRule& skip)
{
    const bool out_side = dot(dir, sf.n) >= 0.0f;
    origin = offsetOrigin(sf.p, out_side ? sf.n : -sf.n);
    skip.object_pos = sf.obj_pos;
    skip.tri_pos = sf.tri_pos;
    skip.light_object_pos = kNoPrim;
    if (sf.is_sphere) {
        // Leaving on the side the ray came from is outward exactly when it hit the outside.
        skip.sphere_mode = (out_side == sf.front) ? kSphereSkipAll : kSphereFarOnly;
    } else {
        skip.sphere_mode = kSphereTestBoth;
    }
}

} // namespace albedo_b200
