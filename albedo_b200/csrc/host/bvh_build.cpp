// Binned-SAH BVH build; each helper restates the accel/bvh.cpp function named beside it.
#include "bvh_build.hpp"

#include <algorithm>
#include <array>
#include <cstddef>
#include <exception>
#include <format>
#include <memory>
#include <optional>
#include <stdexcept>
#include <thread>
#include <utility>

namespace albedo_b200 {

namespace {

constexpr std::size_t kBins{12};            // accel/bvh.cpp:27
constexpr double kTraversalCost{0.125};     // accel/bvh.cpp:30
constexpr std::size_t kMaxLeaf{4};          // accel/bvh.cpp:32
constexpr std::size_t kSahDepthLimit{32};   // accel/bvh.cpp:35

struct Prim {
    Box3 bounds{};
    Vec3 centroid{};
    std::size_t index{};
};

// centroidOf, accel/bvh.cpp:45-50: halved before adding.
Vec3 centroidOf(const Box3& box)
{
    return {box.min.x / 2 + box.max.x / 2, box.min.y / 2 + box.max.y / 2, box.min.z / 2 + box.max.z / 2};
}

struct Extents {
    Box3 bounds{};
    Box3 centroids{};
};

// Ranges of at least this many primitives are scanned on several threads.
constexpr std::size_t kParallelScanMinimum{1 << 17};

// Runs scan(chunk, range) over `chunks` contiguous pieces of `prims`, each on its
// own thread (the first on the calling one).
template <typename F>
void scanChunks(std::span<const Prim> prims, unsigned chunks, F&& scan)
{
    const auto piece = [&](unsigned c) {
        const std::size_t begin{prims.size() * c / chunks};
        const std::size_t end{prims.size() * (c + 1) / chunks};
        return prims.subspan(begin, end - begin);
    };
    // A jthread joins when destroyed, so an exception that leaves early (a
    // thread that fails to start, or the calling thread's own share) still
    // waits for the workers already running.
    std::vector<std::jthread> workers;
    for (unsigned c{1}; c < chunks; ++c) {
        workers.emplace_back([&, c] { scan(c, piece(c)); });
    }
    scan(0u, piece(0));
    for (std::jthread& worker : workers) {
        worker.join();
    }
}

unsigned scanThreads(std::size_t count, unsigned threads)
{
    return count < kParallelScanMinimum ? 1u : threads;
}

// extentsOf, accel/bvh.cpp:70-78. Boxes merge by minimum and maximum, which
// give the same result in any order, so large ranges merge per thread first.
Extents extentsOf(std::span<const Prim> prims, unsigned threads = 1)
{
    const unsigned chunks{scanThreads(prims.size(), threads)};
    std::vector<Extents> parts(chunks);
    scanChunks(prims, chunks, [&](unsigned c, std::span<const Prim> range) {
        Extents e;
        for (const Prim& p : range) {
            e.bounds = merged(e.bounds, p.bounds);
            e.centroids = merged(e.centroids, p.centroid);
        }
        parts[c] = e;
    });
    Extents e;
    for (const Extents& part : parts) {
        e.bounds = merged(e.bounds, part.bounds);
        e.centroids = merged(e.centroids, part.centroids);
    }
    return e;
}

// widestAxis, accel/bvh.cpp:80-87.
std::size_t widestAxis(const Box3& box)
{
    const Vec3 extent{box.extent()};
    if (extent.x >= extent.y && extent.x >= extent.z) {
        return 0;
    }
    return extent.y >= extent.z ? 1 : 2;
}

// halfDistance / halfSpread, accel/bvh.cpp:91-100.
double halfDistance(double low, double high) { return high / 2 - low / 2; }
double halfSpread(const Box3& centroids, std::size_t axis)
{
    return halfDistance(axisOf(centroids.min, axis), axisOf(centroids.max, axis));
}

// binOf, accel/bvh.cpp:107-118.
std::size_t binOf(Vec3 centroid, const Box3& centroids, std::size_t axis)
{
    const double low{axisOf(centroids.min, axis)};
    const double fraction{halfDistance(low, axisOf(centroid, axis)) / halfSpread(centroids, axis)};
    const double limited{fraction > 0 ? std::min(fraction, 1.0) : 0.0};
    const double scaled{limited * static_cast<double>(kBins)};
    return std::min(static_cast<std::size_t>(scaled), kBins - 1);
}

struct Bin {
    Box3 bounds{};
    std::size_t count{};
};

struct Split {
    std::size_t axis{};
    std::size_t last_left_bin{};
    double cost{std::numeric_limits<double>::infinity()};
};

// bestSplitAlong, accel/bvh.cpp:134-160: bin, sweep from the right, then scan
// left. A bin is a box merge and a count, so large ranges bin per thread and
// the per-thread bins merge into the same bins.
Split bestSplitAlong(std::span<const Prim> prims, const Extents& extents, std::size_t axis, unsigned threads)
{
    const unsigned chunks{scanThreads(prims.size(), threads)};
    std::vector<std::array<Bin, kBins>> parts(chunks);
    scanChunks(prims, chunks, [&](unsigned c, std::span<const Prim> range) {
        std::array<Bin, kBins> part{};
        for (const Prim& p : range) {
            Bin& bin{part[binOf(p.centroid, extents.centroids, axis)]};
            bin.bounds = merged(bin.bounds, p.bounds);
            ++bin.count;
        }
        parts[c] = part;
    });
    std::array<Bin, kBins> bins{};
    for (const auto& part : parts) {
        for (std::size_t k{0}; k < kBins; ++k) {
            bins[k] = {merged(bins[k].bounds, part[k].bounds), bins[k].count + part[k].count};
        }
    }
    std::array<Bin, kBins> right_of{};
    for (std::size_t bin{kBins - 1}; bin > 0; --bin) {
        const Bin next{bin + 1 < kBins ? right_of[bin] : Bin{}};
        right_of[bin - 1] = {merged(next.bounds, bins[bin].bounds), next.count + bins[bin].count};
    }
    Split best{.axis = axis};
    Bin left{};
    for (std::size_t bin{0}; bin + 1 < kBins; ++bin) {
        left = {merged(left.bounds, bins[bin].bounds), left.count + bins[bin].count};
        const Bin& right{right_of[bin]};
        const double cost{left.bounds.surfaceArea() * static_cast<double>(left.count) +
                          right.bounds.surfaceArea() * static_cast<double>(right.count)};
        if (cost < best.cost) {
            best = {.axis = axis, .last_left_bin = bin, .cost = cost};
        }
    }
    return best;
}

// bestSplit, accel/bvh.cpp:163-176.
std::optional<Split> bestSplit(std::span<const Prim> prims, const Extents& extents, unsigned threads)
{
    std::optional<Split> best;
    for (std::size_t axis{0}; axis < 3; ++axis) {
        if (!(halfSpread(extents.centroids, axis) > 0)) {
            continue;
        }
        const Split split{bestSplitAlong(prims, extents, axis, threads)};
        if (!best || split.cost < best->cost) {
            best = split;
        }
    }
    return best;
}

struct Partition {
    std::size_t left_count{};
    std::size_t axis{};
};

// partitionForSplit, accel/bvh.cpp:186-220.
Partition partitionForSplit(std::span<Prim> prims, const Extents& extents, std::size_t depth, unsigned threads = 1)
{
    const std::size_t count{prims.size()};
    if (depth < kSahDepthLimit) {
        if (const auto split{bestSplit(prims, extents, threads)}) {
            const double area{extents.bounds.surfaceArea()};
            const bool leaf_is_cheaper{static_cast<double>(count) * area <= kTraversalCost * area + split->cost};
            if (count <= kMaxLeaf && leaf_is_cheaper) {
                return {};
            }
            const auto middle{std::partition(prims.begin(), prims.end(), [&](const Prim& p) {
                return binOf(p.centroid, extents.centroids, split->axis) <= split->last_left_bin;
            })};
            return {static_cast<std::size_t>(middle - prims.begin()), split->axis};
        }
    }
    if (count <= kMaxLeaf) {
        return {};
    }
    const std::size_t axis{widestAxis(extents.centroids)};
    const std::size_t half{count / 2};
    const auto middle{prims.begin() + static_cast<std::ptrdiff_t>(half)};
    std::nth_element(prims.begin(), middle, prims.end(), [&](const Prim& a, const Prim& b) {
        return axisOf(a.centroid, axis) < axisOf(b.centroid, axis);
    });
    return {half, axis};
}

// buildSubtree, accel/bvh.cpp:224-244 (recursion depth is bounded by 32 + log2 n).
// Appends the subtree to `nodes`; interior offsets index `nodes` itself.
std::size_t buildSubtree(std::vector<BuildNode>& nodes, std::uint32_t& max_depth, std::span<Prim> prims,
                         std::size_t first, std::size_t depth)
{
    const std::size_t index{nodes.size()};
    const Extents extents{extentsOf(prims)};
    nodes.push_back({.bounds = extents.bounds});
    max_depth = std::max<std::uint32_t>(max_depth, static_cast<std::uint32_t>(depth));
    const Partition partition{prims.size() == 1 ? Partition{} : partitionForSplit(prims, extents, depth)};
    if (partition.left_count == 0) {
        nodes[index].offset = first;
        nodes[index].count = static_cast<std::uint32_t>(prims.size());
        return index;
    }
    buildSubtree(nodes, max_depth, prims.first(partition.left_count), first, depth + 1);
    const std::size_t second{buildSubtree(nodes, max_depth, prims.subspan(partition.left_count),
                                          first + partition.left_count, depth + 1)};
    nodes[index].offset = second;
    nodes[index].axis = static_cast<std::uint8_t>(partition.axis);
    return index;
}

// Ranges below this many primitives are built on one thread.
constexpr std::size_t kParallelMinimum{8192};

// A subtree built in parallel: either nodes built on one thread (interior
// offsets relative to the piece's first node) or one node whose two children
// were built concurrently. Every node makes the same decision from the same
// primitive range as in the one-thread build, because a node's range is
// partitioned before its children start, so the tree is the same.
struct Piece {
    std::vector<BuildNode> nodes;
    BuildNode self{};
    std::unique_ptr<Piece> left;
    std::unique_ptr<Piece> right;
    std::size_t total{0};
    std::uint32_t max_depth{0};
};

std::unique_ptr<Piece> buildPiece(std::span<Prim> prims, std::size_t first, std::size_t depth, unsigned threads)
{
    auto piece{std::make_unique<Piece>()};
    if (threads <= 1 || prims.size() < kParallelMinimum) {
        piece->nodes.reserve(2 * prims.size() - 1);
        buildSubtree(piece->nodes, piece->max_depth, prims, first, depth);
        piece->total = piece->nodes.size();
        return piece;
    }
    const Extents extents{extentsOf(prims, threads)};
    const Partition partition{partitionForSplit(prims, extents, depth, threads)};
    if (partition.left_count == 0) {
        piece->nodes.push_back({.bounds = extents.bounds, .offset = first,
                                .count = static_cast<std::uint32_t>(prims.size())});
        piece->total = 1;
        piece->max_depth = static_cast<std::uint32_t>(depth);
        return piece;
    }
    piece->self = {.bounds = extents.bounds, .axis = static_cast<std::uint8_t>(partition.axis)};
    // Threads split in proportion to the primitives on each side.
    const double share{static_cast<double>(partition.left_count) / static_cast<double>(prims.size())};
    const unsigned left_threads{std::clamp(static_cast<unsigned>(share * threads + 0.5), 1u, threads - 1)};
    std::exception_ptr failure;
    std::thread worker{[&] {
        try {
            piece->left = buildPiece(prims.first(partition.left_count), first, depth + 1, left_threads);
        } catch (...) {
            failure = std::current_exception();
        }
    }};
    try {
        piece->right = buildPiece(prims.subspan(partition.left_count), first + partition.left_count, depth + 1,
                                  threads - left_threads);
    } catch (...) {
        worker.join();
        throw;
    }
    worker.join();
    if (failure) {
        std::rethrow_exception(failure);
    }
    piece->total = 1 + piece->left->total + piece->right->total;
    piece->max_depth = std::max(piece->left->max_depth, piece->right->max_depth);
    return piece;
}

// Lays a piece out in depth-first order from node `at`, collecting the
// one-thread pieces (with their positions) for a parallel copy.
void layOut(const Piece& piece, std::vector<BuildNode>& out, std::size_t at,
            std::vector<std::pair<const Piece*, std::size_t>>& copies)
{
    if (!piece.left) {
        copies.emplace_back(&piece, at);
        return;
    }
    BuildNode self{piece.self};
    self.offset = at + 1 + piece.left->total;
    out[at] = self;
    layOut(*piece.left, out, at + 1, copies);
    layOut(*piece.right, out, at + 1 + piece.left->total, copies);
}

void copyPiece(const Piece& piece, std::vector<BuildNode>& out, std::size_t at)
{
    for (std::size_t i{0}; i < piece.nodes.size(); ++i) {
        BuildNode node{piece.nodes[i]};
        if (node.count == 0) {
            node.offset += at;
        }
        out[at + i] = node;
    }
}

} // namespace

BuiltBvh buildBvh(std::span<const Box3> primitive_bounds, unsigned threads)
{
    BuiltBvh bvh;
    if (primitive_bounds.empty()) {
        return bvh;
    }
    std::vector<Prim> prims;
    prims.reserve(primitive_bounds.size());
    for (std::size_t index{0}; index < primitive_bounds.size(); ++index) {
        const Box3& box{primitive_bounds[index]};
        if (!isFinite(box.min) || !isFinite(box.max) || box.isEmpty()) {
            throw std::invalid_argument{std::format("BVH primitive {} has an empty or non-finite box", index)};
        }
        prims.push_back({box, centroidOf(box), index});
    }
    if (threads == 0) {
        threads = std::max(1u, std::thread::hardware_concurrency());
    }
    std::unique_ptr<Piece> root{buildPiece(prims, 0, 0, threads)};
    bvh.max_depth = root->max_depth;
    if (!root->left) {
        bvh.nodes = std::move(root->nodes);
    } else {
        bvh.nodes.resize(root->total);
        std::vector<std::pair<const Piece*, std::size_t>> copies;
        layOut(*root, bvh.nodes, 0, copies);
        // A jthread joins when destroyed, so an exception that leaves early (a
        // thread that fails to start, or the calling thread's own share) still
        // waits for the workers already running.
        std::vector<std::jthread> workers;
        for (std::size_t t{1}; t < copies.size(); ++t) {
            workers.emplace_back([&, t] { copyPiece(*copies[t].first, bvh.nodes, copies[t].second); });
        }
        copyPiece(*copies[0].first, bvh.nodes, copies[0].second);
        for (std::jthread& worker : workers) {
            worker.join();
        }
    }
    bvh.order.reserve(prims.size());
    for (const Prim& p : prims) {
        bvh.order.push_back(static_cast<std::uint32_t>(p.index));
    }
    return bvh;
}

} // namespace albedo_b200
