// Host check of the traversal's box test (albedo_b200/csrc/kernels/traverse.cuh):
// slabTestOrdered, the branchless form, against slabTest, the clip of the
// reference's clipToSlab restated in FP32 (accel/bvh.hpp:93-114). Both are
// restated here in host FP32 arithmetic, which rounds as the device's _rn
// intrinsics do (built with -ffp-contract=off, no flush to zero); the device's
// three-input max/min skip NaN operands as the fmaxf/fminf chain does.
//
// Prints one line per category: rays, disagreements, and the disagreements that
// are not the documented exception (a -infinite inverse direction component
// and an origin on exactly one of that axis's two box planes, where the clip
// rejects the box, or enters it at +infinity when the range is unbounded, and
// the branchless test enters it).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>

namespace {

constexpr float kW = 1.00000036f;

struct Ray {
    float o[3];
    float inv[3];
};

struct Box {
    float lo[3];
    float hi[3];
};

// slabTest: clipToSlab on three axes (swap when near > far, widen the exit,
// keep the range when a distance is NaN).
bool clip(const Box& b, const Ray& r, float tmin, float tmax, float& entry)
{
    float lo = tmin;
    float hi = tmax;
    for (int a = 0; a < 3; ++a) {
        float n = (b.lo[a] - r.o[a]) * r.inv[a];
        float f = (b.hi[a] - r.o[a]) * r.inv[a];
        if (n > f) {
            const float s = n;
            n = f;
            f = s;
        }
        f *= f < 0.0f ? 2.0f - kW : kW;
        lo = n > lo ? n : lo;
        hi = f < hi ? f : hi;
    }
    entry = lo;
    return lo <= hi;
}

// slabTestOrdered with the near and far planes picked by the inverse's sign bit.
bool ordered(const Box& b, const Ray& r, float tmin, float tmax, float& entry)
{
    float tn[3];
    float tf[3];
    for (int a = 0; a < 3; ++a) {
        const bool neg = std::signbit(r.inv[a]);
        const float nearp = neg ? b.hi[a] : b.lo[a];
        const float farp = neg ? b.lo[a] : b.hi[a];
        tn[a] = (nearp - r.o[a]) * r.inv[a];
        tf[a] = (farp - r.o[a]) * r.inv[a];
    }
    const float lo = std::fmax(std::fmax(tn[0], tn[1]), std::fmax(tn[2], tmin));
    const float f = std::fmin(std::fmin(tf[0], tf[1]), tf[2]);
    const float hi = std::fmin(std::fmax(f * kW, f * (2.0f - kW)), tmax);
    entry = lo;
    return lo <= hi;
}

// The documented exception: on some axis the inverse is -infinite and the
// origin lies on exactly one of the box's two planes.
bool exception(const Box& b, const Ray& r)
{
    for (int a = 0; a < 3; ++a) {
        if (std::isinf(r.inv[a]) && r.inv[a] < 0.0f) {
            const bool on_lo = r.o[a] == b.lo[a];
            const bool on_hi = r.o[a] == b.hi[a];
            if (on_lo != on_hi) {
                return true;
            }
        }
    }
    return false;
}

struct Tally {
    long rays = 0;
    long differ = 0;
    long unexplained = 0;
    long entered_more = 0;
    long hits = 0;
};

void compare(Tally& t, const Box& b, const Ray& r, float tmin, float tmax)
{
    float e1 = 0.0f;
    float e2 = 0.0f;
    const bool h1 = clip(b, r, tmin, tmax, e1);
    const bool h2 = ordered(b, r, tmin, tmax, e2);
    ++t.rays;
    t.hits += h1 ? 1 : 0;
    // Entry distances compare as values: a zero's sign is not read.
    const bool same = h1 == h2 && (!h1 || e1 == e2 || (std::isnan(e1) && std::isnan(e2)));
    if (same) {
        return;
    }
    ++t.differ;
    // The exception: the clip's NaN rejects the box, or, over an unbounded range,
    // leaves its entry distance at +infinity; the branchless test enters it at
    // the other axes' entry.
    if (h2 && (!h1 || std::isinf(e1)) && exception(b, r)) {
        ++t.entered_more;
        return;
    }
    ++t.unexplained;
    if (t.unexplained <= 3) {
        std::fprintf(stderr, "unexplained: clip %d %.9g ordered %d %.9g\n", h1, e1, h2, e2);
    }
}

float pick(std::mt19937_64& g, const float* values, int n)
{
    return values[std::uniform_int_distribution<int>(0, n - 1)(g)];
}

} // namespace

int main()
{
    std::mt19937_64 g(12345);
    std::uniform_real_distribution<float> u(-4.0f, 4.0f);
    std::uniform_real_distribution<float> ext(0.0f, 2.0f);
    const float tmaxes[] = {INFINITY, 1e30f, 10.0f, 2.5f, 0.5f};

    // Ordinary rays: random boxes, origins and directions (finite inverses).
    Tally finite;
    for (int i = 0; i < 2000000; ++i) {
        Box b;
        Ray r;
        for (int a = 0; a < 3; ++a) {
            b.lo[a] = u(g);
            b.hi[a] = b.lo[a] + ext(g);
            r.o[a] = u(g);
            float d = u(g);
            if (d == 0.0f) {
                d = 1.0f;
            }
            r.inv[a] = 1.0f / d;
        }
        compare(finite, b, r, 0.0f, tmaxes[i % 5]);
    }

    // Aimed rays: from a random origin toward a random point of the box, so most
    // of them enter it; entries and exits at every range bound.
    Tally aimed;
    std::uniform_real_distribution<float> unit(0.0f, 1.0f);
    for (int i = 0; i < 2000000; ++i) {
        Box b;
        Ray r;
        for (int a = 0; a < 3; ++a) {
            b.lo[a] = u(g);
            b.hi[a] = b.lo[a] + ext(g);
            r.o[a] = 3.0f * u(g);
            const float target = b.lo[a] + unit(g) * (b.hi[a] - b.lo[a]);
            float d = target - r.o[a];
            if (d == 0.0f) {
                d = 1e-3f;
            }
            r.inv[a] = 1.0f / d;
        }
        compare(aimed, b, r, 0.0f, tmaxes[i % 5]);
    }

    // Degenerate rays: coordinates from a small set, so origins land on box
    // planes; direction components among +-0, subnormals, tiny, huge and
    // ordinary values (infinite or huge inverses); boxes with infinite bounds.
    const float coords[] = {-1.0f, -0.5f, 0.0f, -0.0f, 0.5f, 1.0f, 2.0f, 0x1p-126f, -0x1p-130f};
    const float bounds[] = {-1.0f, -0.5f, 0.0f, 0.5f, 1.0f, 2.0f, -INFINITY, INFINITY, 0x1p-126f};
    const float dirs[] = {0.0f, -0.0f, 0x1p-140f, -0x1p-140f, 0x1p-127f, -0x1p-127f, 1.0f, -1.0f, 0.25f,
                          -3.0f, 3e38f, -3e38f};
    Tally degenerate;
    for (int i = 0; i < 4000000; ++i) {
        Box b;
        Ray r;
        for (int a = 0; a < 3; ++a) {
            float x = pick(g, bounds, 9);
            float y = pick(g, bounds, 9);
            if (x > y) {
                const float s = x;
                x = y;
                y = s;
            }
            b.lo[a] = x;
            b.hi[a] = y;
            r.o[a] = pick(g, coords, 9);
            r.inv[a] = 1.0f / pick(g, dirs, 12);
        }
        compare(degenerate, b, r, i % 3 == 0 ? 0.0f : 1e-4f, tmaxes[i % 5]);
    }

    std::printf("finite rays=%ld hits=%ld differ=%ld unexplained=%ld\n", finite.rays, finite.hits, finite.differ,
                finite.unexplained);
    std::printf("aimed rays=%ld hits=%ld differ=%ld unexplained=%ld\n", aimed.rays, aimed.hits, aimed.differ,
                aimed.unexplained);
    std::printf("degenerate rays=%ld hits=%ld differ=%ld unexplained=%ld entered_more=%ld\n", degenerate.rays,
                degenerate.hits, degenerate.differ, degenerate.unexplained, degenerate.entered_more);
    return 0;
}
