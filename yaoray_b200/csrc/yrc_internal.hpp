// Internal host-side helpers shared by the libyrcuda translation units.
#pragma once

#include "yrcuda.h"

#include <cstdint>
#include <string>
#include <vector>

namespace yrc {

// Records `message` as this thread's last error and returns `status`.
yrc_status Fail(yrc_status status, const std::string& message);
// Clears this thread's last error and returns YRC_OK.
yrc_status Ok();

struct Vec3 {
    float x = 0.0f, y = 0.0f, z = 0.0f;
};

// Bounds3f (include/yaoray/core/bounds.hpp:12-25): an empty box is
// (+inf, -inf) so the first union takes the operand.
struct Box {
    Vec3 lo{__builtin_inff(), __builtin_inff(), __builtin_inff()};
    Vec3 hi{-__builtin_inff(), -__builtin_inff(), -__builtin_inff()};
};

// Host copy of one RenderBvh (bvh.hpp:72-81).
struct HostBvh {
    std::vector<yrc_bvh_node> nodes;
    std::vector<int32_t> primitive_indices;
    std::vector<yrc_bvh_primitive> primitives;
    int32_t max_depth = 0;
    int32_t total_triangles = 0;
    int32_t total_spheres = 0;
};

yrc_bvh_view ViewOf(const HostBvh& bvh);

// Position of vertex `i` of a yrc_geometry.
inline const float* VertexPosition(const yrc_geometry& g, uint64_t i) {
    return reinterpret_cast<const float*>(reinterpret_cast<const char*>(g.positions) +
                                          static_cast<int64_t>(i) * g.vertex_stride);
}

// One object handed to the hierarchy builder: a triangle, a sphere, or (for
// the TLAS) an instance's world box.
struct BuildRef {
    int32_t flat_index;
    Box bounds;
    Vec3 centroid;
};

// Builds the binary hierarchy over `refs` (reordered in place) into `bvh`'s
// nodes / primitive_indices / max_depth. Returns false with `error` set on a
// build error.
bool BuildHierarchy(std::vector<BuildRef>& refs, const yrc_bvh_options& options, HostBvh& bvh,
                    std::string& error);

// Builds a flat BVH (primitives + hierarchy) over a geometry's triangles and
// spheres, as BuildBvh does; with `device`, the hierarchy is built on the
// current CUDA device (BuildHierarchyDevice) unless that reports a range it
// leaves to the host, and *on_device (optional) tells which happened.
bool BuildFlatBvh(const yrc_geometry& geometry, const yrc_bvh_options& options, HostBvh& bvh,
                  std::string& error, bool device = false, bool* on_device = nullptr);

// The reference's MedianPartition (bvh_split_policy.cpp:98-113) of a whole
// range held as its own vector: std::nth_element by centroid on the range's
// widest centroid axis at mid = size / 2. The device builder asks the host
// for it on degenerate ranges, so its permutation is the standard library's
// own, as in the reference.
void MedianPartitionRange(std::vector<BuildRef>& refs);

// The host builder's serial build of a whole range (refs permuted to slot
// order) as one subtree rooted at `depth`: nodes with subtree-local indices
// (an interior node's payload is its right child's local index, a leaf's its
// first slot relative to the range). For device subtrees that meet a median
// split. Returns false with `error` set on a build error.
bool BuildSubtreeHost(std::vector<BuildRef>& refs, const yrc_bvh_options& options, int depth,
                      std::vector<yrc_bvh_node>& nodes, int32_t& max_depth, std::string& error);

// The hierarchy of BuildHierarchy built on the current CUDA device, byte for
// byte the same. Returns 1 when built, 0 when a range needs the median split
// (std::nth_element) or the options ask for median splits — the caller then
// builds on the host — and -1 on a device error (`error` set). `refs` are
// not reordered.
int BuildHierarchyDevice(std::vector<BuildRef>& refs, const yrc_bvh_options& options, HostBvh& bvh,
                         std::string& error);

// The whole flat build on the current CUDA device: refs and primitives from
// the geometry (uploaded), then the hierarchy; same return convention (0 for
// median splits and for invalid geometry, which the host build reports).
int BuildFlatDevice(const yrc_geometry& geometry, const yrc_bvh_options& options, HostBvh& bvh,
                    std::string& error);

}  // namespace yrc
