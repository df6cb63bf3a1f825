// Binned-SAH BVH construction that reproduces the reference's trees exactly.
//
// The device traverses the same topology the reference CPU renderer does, so hit
// ids agree on ties and node-visit counts are comparable. The build restates
// accel/bvh.cpp:19-270: 12 bins, traversal cost 0.125, leaves of at most 4
// primitives, SAH splits above depth 32 and median splits below, std::partition
// for SAH splits and std::nth_element for median splits (the same libstdc++
// algorithms, so equal inputs give equal permutations), nodes in depth-first
// order with the first child right after its parent.
#pragma once

#include "host_math.hpp"

#include <cstdint>
#include <span>
#include <vector>

namespace albedo_b200 {

// One node in depth-first order (accel/bvh.hpp:36-46).
struct BuildNode {
    Box3 bounds{};
    // Leaf: first position in `order`. Interior: index of the second child.
    std::uint64_t offset{};
    // Primitives in a leaf; 0 marks an interior node.
    std::uint32_t count{};
    // Interior: split axis 0, 1 or 2.
    std::uint8_t axis{};
};

struct BuiltBvh {
    std::vector<BuildNode> nodes;
    // Primitive indices in leaf order.
    std::vector<std::uint32_t> order;
    // Deepest node, counting the root as depth 0.
    std::uint32_t max_depth{0};
};

// Builds over boxes 0..n-1. Throws std::invalid_argument for an empty or
// non-finite box, as accel/bvh.cpp:253-261 does. Subtrees of large ranges are
// built on up to `threads` threads (0: one per hardware thread); the tree is
// the same for every thread count.
BuiltBvh buildBvh(std::span<const Box3> primitive_bounds, unsigned threads = 0);

} // namespace albedo_b200
