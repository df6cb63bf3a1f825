// The BVH build gives the same tree on any number of threads: nodes (bounds bit
// for bit, offsets, counts, axes), leaf order and depth, on seeded box sets that
// reach every branch of the build: SAH splits, leaves chosen by cost, median
// splits (coincident centroids, and depth beyond the SAH limit), and ranges on
// both sides of the parallel threshold. Prints one line per case.
#include "host/bvh_build.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

using namespace albedo_b200;

namespace {

bool sameTree(const BuiltBvh& a, const BuiltBvh& b)
{
    if (a.nodes.size() != b.nodes.size() || a.order != b.order || a.max_depth != b.max_depth) {
        return false;
    }
    for (std::size_t i{0}; i < a.nodes.size(); ++i) {
        const BuildNode& x{a.nodes[i]};
        const BuildNode& y{b.nodes[i]};
        if (std::memcmp(&x.bounds, &y.bounds, sizeof(Box3)) != 0 || x.offset != y.offset || x.count != y.count ||
            x.axis != y.axis) {
            return false;
        }
    }
    return true;
}

Box3 box(Vec3 c, double half) { return {{c.x - half, c.y - half, c.z - half}, {c.x + half, c.y + half, c.z + half}}; }

std::vector<Box3> uniformBoxes(std::size_t n, unsigned seed)
{
    std::mt19937_64 rng{seed};
    std::uniform_real_distribution<double> u{-100.0, 100.0};
    std::uniform_real_distribution<double> s{0.01, 2.0};
    std::vector<Box3> boxes;
    for (std::size_t i{0}; i < n; ++i) {
        boxes.push_back(box({u(rng), u(rng), u(rng)}, s(rng)));
    }
    return boxes;
}

std::vector<Box3> clusteredBoxes(std::size_t n, unsigned seed)
{
    std::mt19937_64 rng{seed};
    std::normal_distribution<double> g{0.0, 1.0};
    std::uniform_int_distribution<int> pick{0, 4};
    const Vec3 centers[5]{{0, 0, 0}, {50, 0, 0}, {0, 80, 0}, {0, 0, -30}, {1e3, 1e3, 1e3}};
    std::vector<Box3> boxes;
    for (std::size_t i{0}; i < n; ++i) {
        const Vec3 c{centers[pick(rng)]};
        const double half{i % 997 == 0 ? 500.0 : 0.05};
        boxes.push_back(box({c.x + g(rng), c.y + g(rng), c.z + g(rng)}, half));
    }
    return boxes;
}

std::vector<Box3> coincidentBoxes(std::size_t n)
{
    std::vector<Box3> boxes;
    for (std::size_t i{0}; i < n; ++i) {
        boxes.push_back(box({1.0, 2.0, 3.0}, 0.5 + static_cast<double>(i % 7)));
    }
    return boxes;
}

// Centroids at 2^-k along x: each SAH split peels off the far end, so the tree
// passes the SAH depth limit and the lower levels split at the median.
std::vector<Box3> geometricBoxes(std::size_t n)
{
    std::vector<Box3> boxes;
    for (std::size_t i{0}; i < n; ++i) {
        const double x{std::ldexp(1.0, -static_cast<int>(i % 900))};
        boxes.push_back(box({x, static_cast<double>(i / 900), 0.0}, x * 0.25 + 1e-300));
    }
    return boxes;
}

void check(const char* name, const std::vector<Box3>& boxes)
{
    const BuiltBvh one{buildBvh(boxes, 1)};
    bool same{true};
    for (const unsigned threads : {2u, 3u, 8u, 16u}) {
        same = same && sameTree(one, buildBvh(boxes, threads));
    }
    std::printf("%s n=%zu nodes=%zu depth=%u same=%d\n", name, boxes.size(), one.nodes.size(), one.max_depth,
                same ? 1 : 0);
}

} // namespace

int main()
{
    check("uniform", uniformBoxes(200000, 1));
    check("clustered", clusteredBoxes(100000, 2));
    check("coincident", coincidentBoxes(50000));
    check("geometric", geometricBoxes(40000));
    for (const std::size_t n : {1u, 5u, 8191u, 8192u, 8193u, 16385u}) {
        char name[32];
        std::snprintf(name, sizeof name, "small%zu", n);
        check(name, uniformBoxes(n, static_cast<unsigned>(n)));
    }
    return 0;
}
