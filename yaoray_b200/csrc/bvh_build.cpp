// Host-side binned-SAH BVH builder producing the reference's RenderBvh layout.
//
// The GPU kernels consume "the same SAH BVH layout from src/accel": a binary
// tree of 32-byte RenderBvhNode in depth-first pre-order (left child at
// index + 1, right child in payload_offset), leaf primitive slots appended
// left to right, and RenderBvhPrimitive entries in reference order. To be a
// drop-in the builder must emit exactly the bytes the reference builder does
// (src/accel/bvh_builder.cpp:269-286), so every decision below reproduces the
// reference's floating-point expressions and tie rules:
//   * primitive refs and flat_triangle_index    bvh_builder.cpp:144-238
//   * range bounds (first minimum wins)         bvh_builder_common.cpp:71-88
//   * 12-bucket SAH, cost 0.5 + (nL*AL+nR*AR)/A bvh_split_policy.cpp:123-210
//   * partition / median fallbacks              bvh_split_policy.cpp:212-296
//   * leaf emission and max_depth               bvh_builder_common.cpp:53-69
// The partitions use the same standard-library algorithms (std::partition,
// std::nth_element) with the same predicates, so the element order after each
// split is the same permutation.
//
// Parallelism is a fork-join over subtrees: above a size threshold the left
// subtree is built on a worker into its own node list and spliced in after
// the right one finishes; the splice rebases child and slot offsets, which
// keeps the pre-order layout identical to a serial build.
#include "yrc_internal.hpp"

#include <algorithm>
#include <cmath>
#include <future>
#include <thread>

namespace yrc {
namespace {

constexpr int kBuckets = 12;              // SahBucketCount
constexpr float kTraversalCost = 0.5f;    // SahTraversalCost
constexpr float kDegenerateExtent = 1.0e-8f;

// std::min / std::max argument order matters for the sign of zero: the
// reference keeps the accumulated operand unless the new one is strictly
// smaller (larger).
inline float MinKeep(float acc, float x) { return x < acc ? x : acc; }
inline float MaxKeep(float acc, float x) { return acc < x ? x : acc; }

inline Box Merge(const Box& a, const Box& b) {
    Box r;
    r.lo = {MinKeep(a.lo.x, b.lo.x), MinKeep(a.lo.y, b.lo.y), MinKeep(a.lo.z, b.lo.z)};
    r.hi = {MaxKeep(a.hi.x, b.hi.x), MaxKeep(a.hi.y, b.hi.y), MaxKeep(a.hi.z, b.hi.z)};
    return r;
}

inline Box Grow(const Box& a, const Vec3& p) {
    Box r;
    r.lo = {MinKeep(a.lo.x, p.x), MinKeep(a.lo.y, p.y), MinKeep(a.lo.z, p.z)};
    r.hi = {MaxKeep(a.hi.x, p.x), MaxKeep(a.hi.y, p.y), MaxKeep(a.hi.z, p.z)};
    return r;
}

inline float Comp(const Vec3& v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

inline Vec3 Extent(const Box& b) { return {b.hi.x - b.lo.x, b.hi.y - b.lo.y, b.hi.z - b.lo.z}; }

inline bool Finite(const Vec3& v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }
inline bool Finite(const Box& b) { return Finite(b.lo) && Finite(b.hi); }

inline float HalfArea2(const Box& b) {
    if (b.lo.x > b.hi.x || b.lo.y > b.hi.y || b.lo.z > b.hi.z) return 0.0f;
    const Vec3 e = Extent(b);
    return 2.0f * (e.x * e.y + e.y * e.z + e.z * e.x);
}

inline int WidestAxis(const Box& b) {
    const Vec3 e = Extent(b);
    if (e.x >= e.y && e.x >= e.z) return 0;
    if (e.y >= e.z) return 1;
    return 2;
}

inline int BucketOf(float c, float lo, float extent) {
    const float offset = (c - lo) / extent;
    return std::clamp(static_cast<int>(offset * static_cast<float>(kBuckets)), 0, kBuckets - 1);
}

struct SplitChoice {
    bool leaf = true;
    int mid = -1;
};

// Subtree output: nodes with subtree-local indices, slots local to the subtree.
struct Subtree {
    std::vector<yrc_bvh_node> nodes;
    std::vector<int32_t> slots;
    int32_t max_depth = 0;
};

class HierarchyBuilder {
public:
    HierarchyBuilder(std::vector<BuildRef>& refs, const yrc_bvh_options& options)
        : refs_(refs), options_(options) {
        int threads = options.thread_count;
        if (threads <= 0) {
            threads = static_cast<int>(std::thread::hardware_concurrency());
            if (threads <= 0) threads = 1;
        }
        fork_budget_ = threads;
    }

    bool Run(HostBvh& bvh, std::string& error) {
        Subtree root;
        const int r = Build(0, static_cast<int>(refs_.size()), 1, fork_budget_, root);
        if (r != 0 || !error_.empty()) {
            error = error_.empty() ? "BVH build produced an empty primitive range" : error_;
            return false;
        }
        bvh.nodes = std::move(root.nodes);
        bvh.primitive_indices = std::move(root.slots);
        bvh.max_depth = root.max_depth;
        return true;
    }

    // Builds the whole of refs_ serially as one subtree rooted at `depth`
    // (a range of the device builder): subtree-local node indices, leaf
    // payloads relative to the range.
    bool RunSubtree(int depth, Subtree& out, std::string& error) {
        const int r = Build(0, static_cast<int>(refs_.size()), depth, 1, out);
        if (r != 0 || !error_.empty()) {
            error = error_.empty() ? "BVH build produced an empty primitive range" : error_;
            return false;
        }
        return true;
    }

private:
    void SetError(const char* message) {
        std::lock_guard<std::mutex> lock(error_mutex_);
        if (error_.empty()) error_ = message;
    }

    bool RangeBounds(int begin, int end, Box& node_box, Box& centroid_box) {
        for (int i = begin; i < end; ++i) {
            node_box = Merge(node_box, refs_[i].bounds);
            centroid_box = Grow(centroid_box, refs_[i].centroid);
        }
        if (!Finite(node_box) || !Finite(centroid_box)) {
            SetError("BVH build encountered non-finite primitive bounds");
            return false;
        }
        return true;
    }

    void MedianSplit(int begin, int end, int axis, int mid) {
        std::nth_element(refs_.begin() + begin, refs_.begin() + mid, refs_.begin() + end,
                         [axis](const BuildRef& a, const BuildRef& b) {
                             return Comp(a.centroid, axis) < Comp(b.centroid, axis);
                         });
    }

    SplitChoice Choose(int begin, int end, const Box& node_box, const Box& centroid_box) {
        const int count = end - begin;
        SplitChoice choice;
        if (count <= options_.max_leaf_triangles) return choice;
        choice.leaf = false;
        if (options_.split_method == 1) {
            choice.mid = begin + count / 2;
            MedianSplit(begin, end, WidestAxis(centroid_box), choice.mid);
            return choice;
        }

        int best_axis = -1;
        int best_split = -1;
        float best_cost = __builtin_inff();
        const float parent_area = HalfArea2(node_box);
        if (parent_area > 0.0f) {
            const Vec3 cext = Extent(centroid_box);
            for (int axis = 0; axis < 3; ++axis) {
                const float extent = Comp(cext, axis);
                if (extent < kDegenerateExtent) continue;
                const float lo = Comp(centroid_box.lo, axis);
                int counts[kBuckets] = {};
                Box boxes[kBuckets];
                for (int i = begin; i < end; ++i) {
                    const int b = BucketOf(Comp(refs_[i].centroid, axis), lo, extent);
                    ++counts[b];
                    boxes[b] = Merge(boxes[b], refs_[i].bounds);
                }
                // Prefix (left) and suffix (right) sweeps.
                int left_count[kBuckets];
                Box left_box[kBuckets];
                int right_count[kBuckets];
                Box right_box[kBuckets];
                left_count[0] = counts[0];
                left_box[0] = boxes[0];
                for (int i = 1; i < kBuckets; ++i) {
                    left_count[i] = left_count[i - 1] + counts[i];
                    left_box[i] = Merge(left_box[i - 1], boxes[i]);
                }
                right_count[kBuckets - 1] = counts[kBuckets - 1];
                right_box[kBuckets - 1] = boxes[kBuckets - 1];
                for (int i = kBuckets - 2; i >= 0; --i) {
                    right_count[i] = right_count[i + 1] + counts[i];
                    right_box[i] = Merge(right_box[i + 1], boxes[i]);
                }
                for (int s = 0; s < kBuckets - 1; ++s) {
                    const int nl = left_count[s];
                    const int nr = right_count[s + 1];
                    if (nl == 0 || nr == 0) continue;
                    const float cost = kTraversalCost +
                        (static_cast<float>(nl) * HalfArea2(left_box[s]) +
                         static_cast<float>(nr) * HalfArea2(right_box[s + 1])) / parent_area;
                    if (cost < best_cost) {
                        best_cost = cost;
                        best_axis = axis;
                        best_split = s;
                    }
                }
            }
        }
        const bool found = best_axis >= 0;
        if (found && best_cost >= static_cast<float>(count)) {
            choice.leaf = true;
            return choice;
        }
        choice.mid = begin + count / 2;
        if (!found) {
            MedianSplit(begin, end, WidestAxis(centroid_box), choice.mid);
            return choice;
        }
        const float extent = Comp(Extent(centroid_box), best_axis);
        const float lo = Comp(centroid_box.lo, best_axis);
        const auto it = std::partition(refs_.begin() + begin, refs_.begin() + end,
                                       [best_axis, best_split, lo, extent](const BuildRef& r) {
                                           return BucketOf(Comp(r.centroid, best_axis), lo, extent) <= best_split;
                                       });
        int mid = static_cast<int>(it - refs_.begin());
        if (mid == begin || mid == end) {
            mid = begin + count / 2;
            MedianSplit(begin, end, best_axis, mid);
        }
        choice.mid = mid;
        return choice;
    }

    // Appends `src` (a finished subtree) to `dst`, rebasing its offsets.
    static int32_t Splice(const Subtree& src, Subtree& dst) {
        const int32_t node_base = static_cast<int32_t>(dst.nodes.size());
        const int32_t slot_base = static_cast<int32_t>(dst.slots.size());
        dst.nodes.reserve(dst.nodes.size() + src.nodes.size());
        for (yrc_bvh_node n : src.nodes) {
            if (n.primitive_count > 0) {
                n.payload_offset += slot_base;
            } else if (n.payload_offset >= 0) {
                n.payload_offset += node_base;
            }
            dst.nodes.push_back(n);
        }
        dst.slots.insert(dst.slots.end(), src.slots.begin(), src.slots.end());
        dst.max_depth = std::max(dst.max_depth, src.max_depth);
        return node_base;
    }

    // Builds refs_[begin, end) at `depth` into `out` (appending). Returns the
    // node index in `out`, or -1 on error.
    int Build(int begin, int end, int depth, int budget, Subtree& out) {
        if (begin >= end) {
            SetError("BVH build produced an empty primitive range");
            return -1;
        }
        const int node_index = static_cast<int>(out.nodes.size());
        out.nodes.push_back(yrc_bvh_node{{0, 0, 0}, {0, 0, 0}, -1, 0});

        Box node_box;
        Box centroid_box;
        if (!RangeBounds(begin, end, node_box, centroid_box)) return -1;

        const SplitChoice choice = Choose(begin, end, node_box, centroid_box);
        yrc_bvh_node& self = out.nodes[static_cast<size_t>(node_index)];
        if (choice.leaf) {
            const int32_t first = static_cast<int32_t>(out.slots.size());
            for (int i = begin; i < end; ++i) out.slots.push_back(refs_[i].flat_index);
            self = MakeNode(node_box, first, end - begin);
            out.max_depth = std::max(out.max_depth, depth);
            return node_index;
        }
        if (choice.mid <= begin || choice.mid >= end) {
            SetError("BVH split produced an empty child range");
            return -1;
        }

        int right_child = -1;
        const bool fork = budget > 1 && (end - begin) > options_.parallel_min_subtree_size;
        if (!fork) {
            const int left = Build(begin, choice.mid, depth + 1, 1, out);
            right_child = Build(choice.mid, end, depth + 1, 1, out);
            if (left < 0 || right_child < 0) return -1;
        } else {
            const int left_budget = (budget + 1) / 2;
            Subtree left_tree;
            Subtree right_tree;
            auto left_future = std::async(std::launch::async, [&] {
                return Build(begin, choice.mid, depth + 1, left_budget, left_tree);
            });
            const int r = Build(choice.mid, end, depth + 1, budget - left_budget, right_tree);
            const int l = left_future.get();
            if (l < 0 || r < 0) return -1;
            Splice(left_tree, out);
            right_child = Splice(right_tree, out);
        }
        out.nodes[static_cast<size_t>(node_index)] = MakeNode(node_box, right_child, 0);
        out.max_depth = std::max(out.max_depth, depth);
        return node_index;
    }

    static yrc_bvh_node MakeNode(const Box& b, int32_t payload, int32_t count) {
        yrc_bvh_node n;
        n.bounds_min[0] = b.lo.x;
        n.bounds_min[1] = b.lo.y;
        n.bounds_min[2] = b.lo.z;
        n.bounds_max[0] = b.hi.x;
        n.bounds_max[1] = b.hi.y;
        n.bounds_max[2] = b.hi.z;
        n.payload_offset = payload;
        n.primitive_count = count;
        return n;
    }

    std::vector<BuildRef>& refs_;
    yrc_bvh_options options_;
    int fork_budget_ = 1;
    std::mutex error_mutex_;
    std::string error_;
};

bool ValidOptions(const yrc_bvh_options& o, std::string& error) {
    if (o.max_leaf_triangles < 1) error = "BVH max_leaf_triangles must be at least 1";
    else if (o.thread_count < 0) error = "BVH thread_count must be >= 0";
    else if (o.parallel_min_subtree_size < 1) error = "BVH parallel_min_subtree_size must be >= 1";
    return error.empty();
}

}  // namespace

void MedianPartitionRange(std::vector<BuildRef>& refs) {
    Box centroid_box;
    for (const BuildRef& r : refs) centroid_box = Grow(centroid_box, r.centroid);
    const int axis = WidestAxis(centroid_box);
    const auto mid = refs.begin() + static_cast<std::ptrdiff_t>(refs.size() / 2);
    std::nth_element(refs.begin(), mid, refs.end(), [axis](const BuildRef& a, const BuildRef& b) {
        return Comp(a.centroid, axis) < Comp(b.centroid, axis);
    });
}

bool BuildSubtreeHost(std::vector<BuildRef>& refs, const yrc_bvh_options& options, int depth,
                      std::vector<yrc_bvh_node>& nodes, int32_t& max_depth, std::string& error) {
    yrc_bvh_options serial = options;
    serial.thread_count = 1;
    HierarchyBuilder builder(refs, serial);
    Subtree out;
    if (!builder.RunSubtree(depth, out, error)) return false;
    nodes = std::move(out.nodes);
    max_depth = out.max_depth;
    return true;
}

bool BuildHierarchy(std::vector<BuildRef>& refs, const yrc_bvh_options& options, HostBvh& bvh,
                    std::string& error) {
    if (!ValidOptions(options, error)) return false;
    if (refs.empty()) return true;
    HierarchyBuilder builder(refs, options);
    return builder.Run(bvh, error);
}

bool BuildFlatBvh(const yrc_geometry& g, const yrc_bvh_options& options, HostBvh& bvh,
                  std::string& error, bool device, bool* on_device) {
    if (on_device) *on_device = false;
    if (device) {
        if (!ValidOptions(options, error)) {
            bvh = HostBvh{};
            return false;
        }
        bvh = HostBvh{};
        const int r = BuildFlatDevice(g, options, bvh, error);
        if (r < 0) {
            bvh = HostBvh{};
            return false;
        }
        if (r > 0) {
            if (on_device) *on_device = true;
            return true;
        }
        bvh = HostBvh{};
        error.clear();
    }
    bvh = HostBvh{};
    std::vector<BuildRef> refs;
    refs.reserve(static_cast<size_t>(g.index_count / 3 + g.sphere_count));
    std::vector<yrc_bvh_primitive> prims;
    prims.reserve(refs.capacity());

    int32_t flat_triangle = 0;
    for (int32_t p = 0; p < g.primitive_count; ++p) {
        const yrc_primitive& prim = g.primitives[p];
        const uint64_t first = prim.first_index;
        const uint64_t count = prim.index_count;
        const uint64_t total = static_cast<uint64_t>(g.index_count);
        if (first > total || count > total - first) {
            error = "BVH build encountered a primitive with an invalid index range";
            return false;
        }
        if (count % 3 != 0) {
            error = "BVH build encountered a primitive with a non-triangular index count";
            return false;
        }
        const int32_t tris = static_cast<int32_t>(count / 3);
        for (int32_t t = 0; t < tris; ++t) {
            const uint64_t o = first + static_cast<uint64_t>(t) * 3;
            const uint32_t i0 = g.indices[o], i1 = g.indices[o + 1], i2 = g.indices[o + 2];
            const uint64_t nv = static_cast<uint64_t>(g.vertex_count);
            if (i0 >= nv || i1 >= nv || i2 >= nv) {
                error = "BVH build encountered a triangle with an invalid vertex index";
                return false;
            }
            const float* a = VertexPosition(g, i0);
            const float* b = VertexPosition(g, i1);
            const float* c = VertexPosition(g, i2);
            const Vec3 p0{a[0], a[1], a[2]}, p1{b[0], b[1], b[2]}, p2{c[0], c[1], c[2]};
            Box box;
            box.lo = p0;
            box.hi = p0;
            box = Grow(Grow(box, p1), p2);
            const float third = 1.0f / 3.0f;
            const Vec3 centroid{((p0.x + p1.x) + p2.x) * third, ((p0.y + p1.y) + p2.y) * third,
                                ((p0.z + p1.z) + p2.z) * third};
            if (!Finite(box) || !Finite(centroid)) {
                error = "BVH build encountered non-finite triangle data";
                return false;
            }
            refs.push_back(BuildRef{static_cast<int32_t>(refs.size()), box, centroid});
            prims.push_back(yrc_bvh_primitive{0, p, -1, t, flat_triangle++});
        }
    }
    for (int32_t s = 0; s < g.sphere_count; ++s) {
        const yrc_sphere& sp = g.spheres[s];
        const Vec3 c{sp.center[0], sp.center[1], sp.center[2]};
        const float r = sp.radius;
        Box box;
        box.lo = {c.x - r, c.y - r, c.z - r};
        box.hi = {c.x + r, c.y + r, c.z + r};
        if (!(r > 0.0f) || !Finite(box) || !Finite(c)) {
            error = "BVH build encountered invalid sphere data";
            return false;
        }
        refs.push_back(BuildRef{static_cast<int32_t>(refs.size()), box, c});
        prims.push_back(yrc_bvh_primitive{1, -1, s, -1, -1});
    }

    if (refs.empty()) {
        std::string option_error;
        if (!ValidOptions(options, option_error)) error = option_error;
        return error.empty();
    }
    for (const yrc_bvh_primitive& p : prims) {
        if (p.kind == 0) ++bvh.total_triangles;
        else ++bvh.total_spheres;
    }
    bvh.primitives = std::move(prims);
    if (!BuildHierarchy(refs, options, bvh, error)) {
        bvh = HostBvh{};
        return false;
    }
    return true;
}

yrc_bvh_view ViewOf(const HostBvh& bvh) {
    yrc_bvh_view v;
    v.nodes = bvh.nodes.data();
    v.node_count = static_cast<int64_t>(bvh.nodes.size());
    v.primitive_indices = bvh.primitive_indices.data();
    v.primitive_index_count = static_cast<int64_t>(bvh.primitive_indices.size());
    v.primitives = bvh.primitives.data();
    v.primitive_count = static_cast<int64_t>(bvh.primitives.size());
    v.max_depth = bvh.max_depth;
    return v;
}

}  // namespace yrc

struct yrc_bvh {
    yrc::HostBvh bvh;
};

extern "C" {

void yrc_bvh_options_default(yrc_bvh_options* options) {
    if (!options) return;
    options->split_method = 0;
    options->max_leaf_triangles = 4;
    options->thread_count = 0;
    options->parallel_min_subtree_size = 1024;
}

yrc_status yrc_bvh_build(const yrc_geometry* geometry, const yrc_bvh_options* options, yrc_bvh** out) {
    if (!geometry || !out) return yrc::Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_bvh_build: null argument");
    *out = nullptr;
    yrc_bvh_options opts;
    yrc_bvh_options_default(&opts);
    if (options) opts = *options;
    auto holder = new (std::nothrow) yrc_bvh();
    if (!holder) return yrc::Fail(YRC_ERR_OUT_OF_MEMORY, "yrc_bvh_build: host allocation failed");
    std::string error;
    try {
        if (!yrc::BuildFlatBvh(*geometry, opts, holder->bvh, error)) {
            delete holder;
            return yrc::Fail(YRC_ERR_BUILD, error);
        }
    } catch (const std::exception& e) {
        delete holder;
        return yrc::Fail(YRC_ERR_OUT_OF_MEMORY, std::string("yrc_bvh_build: ") + e.what());
    }
    *out = holder;
    return yrc::Ok();
}

yrc_status yrc_bvh_build_device(const yrc_geometry* geometry, const yrc_bvh_options* options, yrc_bvh** out,
                                int32_t* built_on_device) {
    if (!geometry || !out) return yrc::Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_bvh_build_device: null argument");
    *out = nullptr;
    if (built_on_device) *built_on_device = 0;
    yrc_bvh_options opts;
    yrc_bvh_options_default(&opts);
    if (options) opts = *options;
    auto holder = new (std::nothrow) yrc_bvh();
    if (!holder) return yrc::Fail(YRC_ERR_OUT_OF_MEMORY, "yrc_bvh_build_device: host allocation failed");
    std::string error;
    bool on_device = false;
    try {
        if (!yrc::BuildFlatBvh(*geometry, opts, holder->bvh, error, true, &on_device)) {
            delete holder;
            return yrc::Fail(error.rfind("device BVH build", 0) == 0 ? YRC_ERR_CUDA : YRC_ERR_BUILD, error);
        }
    } catch (const std::exception& e) {
        delete holder;
        return yrc::Fail(YRC_ERR_OUT_OF_MEMORY, std::string("yrc_bvh_build_device: ") + e.what());
    }
    if (built_on_device) *built_on_device = on_device ? 1 : 0;
    *out = holder;
    return yrc::Ok();
}

yrc_status yrc_bvh_get_view(const yrc_bvh* bvh, yrc_bvh_view* view) {
    if (!bvh || !view) return yrc::Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_bvh_get_view: null argument");
    *view = yrc::ViewOf(bvh->bvh);
    return yrc::Ok();
}

void yrc_bvh_destroy(yrc_bvh* bvh) { delete bvh; }

}  // extern "C"
