// Device accelerator: converts the reference's RenderBvh / TwoLevelBvh arrays
// into the traversal layout of device_layout.cuh, uploads it, and runs the
// trace kernels for device- or host-resident ray batches.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cstring>
#include <chrono>
#include <mutex>
#include <string>
#include <vector>

#include "device_layout.cuh"
#include "trace_kernels.hpp"
#include "yrc_internal.hpp"

namespace yrc {
namespace {

constexpr int32_t kUnassigned = INT32_MIN + 1;

struct Layout {
    std::vector<NodePair> pairs;
    std::vector<Record> records;
    std::vector<Instance> instances;
};

Record SkipRecord(int32_t kind) {
    Record r{};
    r.v1.w = IntBits(kind << 1);
    return r;
}

// Builds the traversal records for one BVH. `slot_record` converts one
// primitive slot (an index into primitive_indices) into a Record.
template <typename SlotFn>
bool AddBvh(const yrc_bvh_node* nodes, int64_t node_count, SlotFn slot_record, Layout& out, int32_t& root_ref,
            float root_lo[3], float root_hi[3], int32_t& depth, std::string& error) {
    root_ref = kAbsentRef;
    depth = 0;
    if (node_count <= 0) {
        for (int a = 0; a < 3; ++a) root_lo[a] = root_hi[a] = 0.0f;
        return true;
    }
    for (int a = 0; a < 3; ++a) {
        root_lo[a] = nodes[0].bounds_min[a];
        root_hi[a] = nodes[0].bounds_max[a];
    }
    const size_t n = static_cast<size_t>(node_count);
    std::vector<int32_t> ref(n, kUnassigned);
    std::vector<int32_t> sub_depth(n, 0);
    std::vector<uint8_t> color(n, 0);  // 0 white, 1 on the DFS path, 2 done
    struct Frame {
        int32_t node;
        bool expanded;
    };
    std::vector<Frame> stack;
    stack.push_back({0, false});
    auto child_of = [&](int32_t i, int which) -> int32_t {
        const int64_t c = which == 0 ? static_cast<int64_t>(i) + 1 : nodes[i].payload_offset;
        return (c >= 0 && c < node_count) ? static_cast<int32_t>(c) : -1;
    };
    while (!stack.empty()) {
        Frame& f = stack.back();
        const int32_t i = f.node;
        if (!f.expanded) {
            if (color[i] == 2) {
                stack.pop_back();
                continue;
            }
            color[i] = 1;
            f.expanded = true;
            const yrc_bvh_node& node = nodes[i];
            if (node.primitive_count > 0) {
                const int32_t first = static_cast<int32_t>(out.records.size());
                for (int32_t k = 0; k < node.primitive_count; ++k) {
                    out.records.push_back(slot_record(static_cast<int64_t>(node.payload_offset) + k));
                }
                Record& last = out.records.back();
                last.v1.w = IntBits(FloatBits(last.v1.w) | kRecLast);
                ref[i] = ~first;
                color[i] = 2;
                stack.pop_back();
                continue;
            }
            ref[i] = static_cast<int32_t>(out.pairs.size());
            out.pairs.push_back(NodePair{});
            for (int which = 1; which >= 0; --which) {  // left ends on top
                const int32_t c = child_of(i, which);
                if (c < 0) continue;
                if (color[c] == 1) {
                    error = "BVH node graph contains a cycle";
                    return false;
                }
                if (color[c] == 0) stack.push_back({c, false});
            }
            continue;
        }
        // Post-order: both children have refs now.
        const int32_t l = child_of(i, 0);
        const int32_t r = child_of(i, 1);
        NodePair& p = out.pairs[static_cast<size_t>(ref[i])];
        const float* L = l >= 0 ? nodes[l].bounds_min : nullptr;
        const float* R = r >= 0 ? nodes[r].bounds_min : nullptr;
        float lb[6] = {0, 0, 0, 0, 0, 0}, rb[6] = {0, 0, 0, 0, 0, 0};
        if (L) std::memcpy(lb, L, sizeof(lb));
        if (R) std::memcpy(rb, R, sizeof(rb));
        p.a = make_float4(lb[0], lb[1], lb[2], lb[3]);
        p.b = make_float4(lb[4], lb[5], rb[0], rb[1]);
        p.c = make_float4(rb[2], rb[3], rb[4], rb[5]);
        p.d = make_int4(l >= 0 ? ref[l] : kAbsentRef, r >= 0 ? ref[r] : kAbsentRef, 0, 0);
        int32_t d = 0;
        if (l >= 0) d = std::max(d, sub_depth[l]);
        if (r >= 0) d = std::max(d, sub_depth[r]);
        sub_depth[i] = d + 1;
        color[i] = 2;
        stack.pop_back();
    }
    root_ref = ref[0];
    depth = sub_depth[0];
    return true;
}

// Collapses the binary pairs below `root_ref` into four-wide nodes: starting
// from a pair's two children, the interior entry with the largest box area is
// replaced by its two children until four entries are held or only leaves
// remain. Returns the wide root (node 0, or the leaf / absent root itself)
// and the deepest stack the traversal may need (at most three pushes per
// wide level).
struct WideLayout {
    std::vector<WideNode> nodes;
    int32_t root = kAbsentRef;
    int32_t stack = 1;
};

void BuildWide(const std::vector<NodePair>& pairs, int32_t root_ref, WideLayout& w) {
    w.nodes.clear();
    w.root = root_ref;
    w.stack = 1;
    if (root_ref < 0) return;  // a leaf or an empty root: nothing to collapse
    struct Entry {
        float lo[3], hi[3];
        int32_t ref;
    };
    auto children = [&](int32_t p, Entry out[2]) -> int {
        const NodePair& q = pairs[static_cast<size_t>(p)];
        int n = 0;
        if (q.d.x != kAbsentRef) out[n++] = Entry{{q.a.x, q.a.y, q.a.z}, {q.a.w, q.b.x, q.b.y}, q.d.x};
        if (q.d.y != kAbsentRef) out[n++] = Entry{{q.b.z, q.b.w, q.c.x}, {q.c.y, q.c.z, q.c.w}, q.d.y};
        return n;
    };
    auto area = [](const Entry& e) {
        const float x = e.hi[0] - e.lo[0], y = e.hi[1] - e.lo[1], z = e.hi[2] - e.lo[2];
        return x * y + y * z + z * x;
    };
    struct Work {
        int32_t pair, slot, depth;
    };
    std::vector<Work> work{{root_ref, 0, 1}};
    w.nodes.emplace_back();
    int32_t deepest = 1;
    while (!work.empty()) {
        const Work item = work.back();
        work.pop_back();
        Entry e[4];
        int n = children(item.pair, e);
        for (;;) {
            int best = -1;
            float best_area = -1.0f;
            for (int k = 0; k < n; ++k) {
                if (e[k].ref >= 0 && area(e[k]) > best_area) {
                    best = k;
                    best_area = area(e[k]);
                }
            }
            if (best < 0) break;
            Entry c[2];
            const int m = children(e[best].ref, c);
            if (n - 1 + m > 4) break;
            for (int k = best; k + 1 < n; ++k) e[k] = e[k + 1];  // drop the expanded entry
            --n;
            for (int k = 0; k < m; ++k) e[n++] = c[k];
        }
        WideNode node{};
        float lox[4] = {0, 0, 0, 0}, hix[4] = {0, 0, 0, 0}, loy[4] = {0, 0, 0, 0}, hiy[4] = {0, 0, 0, 0};
        float loz[4] = {0, 0, 0, 0}, hiz[4] = {0, 0, 0, 0};
        int32_t ref[4] = {kAbsentRef, kAbsentRef, kAbsentRef, kAbsentRef};
        for (int k = 0; k < n; ++k) {
            lox[k] = e[k].lo[0], loy[k] = e[k].lo[1], loz[k] = e[k].lo[2];
            hix[k] = e[k].hi[0], hiy[k] = e[k].hi[1], hiz[k] = e[k].hi[2];
            if (e[k].ref >= 0) {
                ref[k] = static_cast<int32_t>(w.nodes.size());
                w.nodes.emplace_back();
                work.push_back({e[k].ref, ref[k], item.depth + 1});
            } else {
                ref[k] = e[k].ref;
            }
        }
        node.lox = make_float4(lox[0], lox[1], lox[2], lox[3]);
        node.hix = make_float4(hix[0], hix[1], hix[2], hix[3]);
        node.loy = make_float4(loy[0], loy[1], loy[2], loy[3]);
        node.hiy = make_float4(hiy[0], hiy[1], hiy[2], hiy[3]);
        node.loz = make_float4(loz[0], loz[1], loz[2], loz[3]);
        node.hiz = make_float4(hiz[0], hiz[1], hiz[2], hiz[3]);
        node.ref = make_int4(ref[0], ref[1], ref[2], ref[3]);
        w.nodes[static_cast<size_t>(item.slot)] = node;
        deepest = std::max(deepest, item.depth);
    }
    w.root = 0;
    w.stack = 3 * deepest + 1;
}

Record TriangleOrSphereRecord(const yrc_geometry& g, const yrc_bvh_view& bvh, int64_t slot) {
    if (slot < 0 || slot >= bvh.primitive_index_count) return SkipRecord(kRecSkip);
    const int32_t pi = bvh.primitive_indices[slot];
    if (pi < 0 || pi >= bvh.primitive_count) return SkipRecord(kRecSkip);
    const yrc_bvh_primitive& p = bvh.primitives[pi];
    Record rec{};
    if (p.kind == 0) {
        if (p.mesh_primitive < 0 || p.mesh_primitive >= g.primitive_count || p.local_triangle < 0) {
            return SkipRecord(kRecSkipCountTriangle);
        }
        const uint32_t base =
            g.primitives[p.mesh_primitive].first_index + static_cast<uint32_t>(p.local_triangle) * 3u;
        if (static_cast<uint64_t>(base) + 2 >= static_cast<uint64_t>(g.index_count)) {
            return SkipRecord(kRecSkipCountTriangle);
        }
        const uint32_t i0 = g.indices[base], i1 = g.indices[base + 1], i2 = g.indices[base + 2];
        const uint64_t nv = static_cast<uint64_t>(g.vertex_count);
        if (i0 >= nv || i1 >= nv || i2 >= nv) return SkipRecord(kRecSkipCountTriangle);
        const float* a = VertexPosition(g, i0);
        const float* b = VertexPosition(g, i1);
        const float* c = VertexPosition(g, i2);
        rec.v0 = make_float4(a[0], a[1], a[2], IntBits(p.flat_triangle_index));
        rec.v1 = make_float4(b[0] - a[0], b[1] - a[1], b[2] - a[2], IntBits(kRecTriangle << 1));
        rec.v2 = make_float4(c[0] - a[0], c[1] - a[1], c[2] - a[2], IntBits(p.mesh_primitive));
        return rec;
    }
    if (p.sphere < 0 || p.sphere >= g.sphere_count) return SkipRecord(kRecSkipCountSphere);
    const yrc_sphere& s = g.spheres[p.sphere];
    rec.v0 = make_float4(s.center[0], s.center[1], s.center[2], IntBits(p.sphere));
    rec.v1 = make_float4(s.radius, 0.0f, 0.0f, IntBits(kRecSphere << 1));
    rec.v2 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    return rec;
}

Record SphereRecord(const yrc_geometry& g, int32_t sphere) {
    if (sphere < 0 || sphere >= g.sphere_count) return SkipRecord(kRecSkipCountSphere);
    const yrc_sphere& s = g.spheres[sphere];
    Record rec{};
    rec.v0 = make_float4(s.center[0], s.center[1], s.center[2], IntBits(sphere));
    rec.v1 = make_float4(s.radius, 0.0f, 0.0f, IntBits(kRecSphere << 1));
    return rec;
}

bool CheckGeometry(const yrc_geometry* g, std::string& error) {
    if (!g) {
        error = "null geometry";
        return false;
    }
    if (g->vertex_count < 0 || g->index_count < 0 || g->primitive_count < 0 || g->sphere_count < 0 ||
        g->instance_count < 0) {
        error = "negative geometry count";
        return false;
    }
    if ((g->vertex_count > 0 && !g->positions) || (g->index_count > 0 && !g->indices) ||
        (g->primitive_count > 0 && !g->primitives) || (g->sphere_count > 0 && !g->spheres) ||
        (g->instance_count > 0 && !g->instances)) {
        error = "null geometry array with a non-zero count";
        return false;
    }
    if (g->vertex_count > 0 && g->vertex_stride < 12) {
        error = "vertex_stride must be at least 12 bytes";
        return false;
    }
    return true;
}

bool CheckBvh(const yrc_bvh_view* b, std::string& error) {
    if (!b) {
        error = "null BVH view";
        return false;
    }
    if (b->node_count < 0 || b->primitive_index_count < 0 || b->primitive_count < 0) {
        error = "negative BVH count";
        return false;
    }
    if ((b->node_count > 0 && !b->nodes) || (b->primitive_index_count > 0 && !b->primitive_indices) ||
        (b->primitive_count > 0 && !b->primitives)) {
        error = "null BVH array with a non-zero count";
        return false;
    }
    return true;
}

}  // namespace

// Host pipeline resources for yrc_trace_host (allocated on first use).
struct HostPipeline {
    static constexpr int kStreams = 4;
    int64_t chunk = 0;
    cudaStream_t streams[kStreams] = {};
    void* d_rays[kStreams] = {};
    void* d_out[kStreams] = {};
    int32_t* d_inst[kStreams] = {};
    uint32_t* d_stats[kStreams] = {};
    unsigned long long* d_counters = nullptr;
};

}  // namespace yrc

struct yrc_accel {
    int device = 0;
    int sm_count = 148;
    yrc::NodePair* d_pairs = nullptr;
    yrc::WideNode* d_wide = nullptr;  // four-wide copy, built on the first yrc_accel_set_wide(1)
    bool wide_enabled = false;
    bool triangles_only = false;  // flat BVH without spheres: a four-wide copy is allowed
    int64_t pair_count = 0;
    yrc::Record* d_records = nullptr;
    yrc::Instance* d_instances = nullptr;
    unsigned long long* d_counter = nullptr;
    int* d_error = nullptr;
    yrc::AccelParams params{};
    int trace_shape[2] = {0, 0};  // launch shape for closest / any hit (autotuned)
    // Launch shape of yrc_trace_host's chunks (closest / any hit), -1: the
    // device shape. Its kernels share the GPU with the chunks' copies, so
    // the fastest device shape need not be the fastest there.
    // Atomic: the host autotuner sets it between its own yrc_trace_host
    // calls, which take the accelerator's lock themselves.
    std::atomic<int> host_shape[2] = {-1, -1};
    int64_t device_bytes = 0;
    yrc::HostPipeline pipe;
    // Ray reordering ahead of device traces (yrc_accel_set_ray_order).
    int order_mode = 0;
    int order_bits = 0;          // 0: chosen from the ray count
    float order_length = 0.05f;  // two-point key distance, fraction of the root box diagonal
    yrc::RayOrderScratch order{};
    int64_t order_capacity = 0;  // rays the key / permutation buffers hold
    int order_hist_bits = 0;     // bins the histogram holds (log2)
    // Per-launch timing of device traces (yrc_accel_set_timing).
    bool timing = false;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    bool timed_order = false;
    std::mutex mutex;
};

namespace yrc {
namespace {

yrc_status CudaFail(cudaError_t err, const char* what) {
    return Fail(err == cudaErrorMemoryAllocation ? YRC_ERR_OUT_OF_MEMORY : YRC_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(err));
}

template <typename T>
cudaError_t Upload(T** dst, const std::vector<T>& src, int64_t& bytes) {
    const size_t n = std::max<size_t>(src.size(), 1);
    cudaError_t err = cudaMalloc(reinterpret_cast<void**>(dst), n * sizeof(T));
    if (err != cudaSuccess) return err;
    bytes += static_cast<int64_t>(n * sizeof(T));
    if (!src.empty()) err = cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
    return err;
}

void FreeAccel(yrc_accel* a) {
    if (!a) return;
    cudaSetDevice(a->device);
    cudaFree(a->d_pairs);
    cudaFree(a->d_wide);
    cudaFree(a->d_records);
    cudaFree(a->d_instances);
    cudaFree(a->d_counter);
    cudaFree(a->d_error);
    HostPipeline& p = a->pipe;
    for (int s = 0; s < HostPipeline::kStreams; ++s) {
        cudaFree(p.d_rays[s]);
        cudaFree(p.d_out[s]);
        cudaFree(p.d_inst[s]);
        cudaFree(p.d_stats[s]);
        if (p.streams[s]) cudaStreamDestroy(p.streams[s]);
    }
    cudaFree(p.d_counters);
    cudaFree(a->order.keys);
    cudaFree(a->order.order);
    cudaFree(a->order.hist);
    cudaFree(a->order.tile_sums);
    for (cudaEvent_t e : a->ev) {
        if (e) cudaEventDestroy(e);
    }
    delete a;
}

// Grows the reordering buffers to `count` rays and 2^bits bins.
cudaError_t EnsureOrderScratch(yrc_accel* a, int64_t count, int bits) {
    cudaError_t err = cudaSuccess;
    if (count > a->order_capacity) {
        cudaFree(a->order.keys);
        cudaFree(a->order.order);
        a->order.keys = a->order.order = nullptr;
        a->order_capacity = 0;
        err = cudaMalloc(reinterpret_cast<void**>(&a->order.keys), static_cast<size_t>(count) * sizeof(uint32_t));
        if (err == cudaSuccess)
            err = cudaMalloc(reinterpret_cast<void**>(&a->order.order), static_cast<size_t>(count) * sizeof(uint32_t));
        if (err != cudaSuccess) return err;
        a->order_capacity = count;
    }
    if (bits > a->order_hist_bits) {
        cudaFree(a->order.hist);
        cudaFree(a->order.tile_sums);
        a->order.hist = a->order.tile_sums = nullptr;
        a->order_hist_bits = 0;
        err = cudaMalloc(reinterpret_cast<void**>(&a->order.hist), (size_t{1} << bits) * sizeof(uint32_t));
        if (err == cudaSuccess)
            err = cudaMalloc(reinterpret_cast<void**>(&a->order.tile_sums),
                             static_cast<size_t>(RayOrderTiles(bits)) * sizeof(uint32_t));
        if (err != cudaSuccess) return err;
        a->order_hist_bits = bits;
    }
    return cudaSuccess;
}

yrc_status Finalize(Layout& layout, int32_t root_ref, const float lo[3], const float hi[3], int32_t two_level,
                    int32_t depth, yrc_accel** out) {
    if (depth + 1 > kMaxTraceStack) {
        return Fail(YRC_ERR_UNSUPPORTED, "BVH too deep for the device traversal stack (" + std::to_string(depth) +
                                             " levels, limit " + std::to_string(kMaxTraceStack - 1) + ")");
    }
    auto* a = new (std::nothrow) yrc_accel();
    if (!a) return Fail(YRC_ERR_OUT_OF_MEMORY, "host allocation failed");
    cudaError_t err = cudaGetDevice(&a->device);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&a->sm_count, cudaDevAttrMultiProcessorCount, a->device);
    if (err == cudaSuccess) err = Upload(&a->d_pairs, layout.pairs, a->device_bytes);
    if (err == cudaSuccess) err = Upload(&a->d_records, layout.records, a->device_bytes);
    a->pair_count = static_cast<int64_t>(layout.pairs.size());
    if (err == cudaSuccess) err = Upload(&a->d_instances, layout.instances, a->device_bytes);
    if (err == cudaSuccess) err = cudaMalloc(reinterpret_cast<void**>(&a->d_counter), sizeof(unsigned long long));
    if (err == cudaSuccess) err = cudaMalloc(reinterpret_cast<void**>(&a->d_error), sizeof(int));
    if (err == cudaSuccess) err = cudaMemset(a->d_error, 0, sizeof(int));
    if (err != cudaSuccess) {
        FreeAccel(a);
        return CudaFail(err, "accelerator upload");
    }
    AccelParams& p = a->params;
    p.pairs = a->d_pairs;
    p.records = a->d_records;
    p.instances = a->d_instances;
    for (int k = 0; k < 3; ++k) {
        p.root_lo[k] = lo[k];
        p.root_hi[k] = hi[k];
    }
    p.root_ref = root_ref;
    p.two_level = two_level;
    p.stack_limit = depth + 1;
    p.wide = nullptr;
    p.wide_root = kAbsentRef;
    p.wide_stack_limit = 0;
    *out = a;
    return Ok();
}

// Rays below this count are traced in the caller's order: sorting them
// costs more than the coherence it buys.
constexpr int64_t kOrderMinRays = int64_t{1} << 16;

// `reorder`: a yrc_trace_device launch, which may sort the rays first (the
// accelerator's reordering buffers are not shared with another stream at
// the time) and records the timing events when timing is on.
yrc_status LaunchInternal(yrc_accel* a, const yrc_ray* rays, int64_t count, int32_t flags, yrc_hit* hits,
                          int32_t* instances, uint8_t* occluded, uint32_t* nt, uint32_t* tt, uint32_t* st,
                          unsigned long long* counter, cudaStream_t stream, bool reorder = false,
                          int shape = -1) {
    if (count <= 0) return Ok();
    TraceArgs args{};
    args.accel = a->params;
    args.rays = reinterpret_cast<const float4*>(rays);
    args.count = count;
    args.hits = hits;
    args.instances = instances;
    args.occluded = occluded;
    args.node_tests = nt;
    args.triangle_tests = tt;
    args.sphere_tests = st;
    args.counter = counter;
    args.error = a->d_error;
    const bool any = (flags & YRC_TRACE_ANY) != 0;
    const bool stats = (flags & YRC_TRACE_STATS) != 0;
    const bool order = reorder && !stats && a->order_mode != kRayOrderOff && count >= kOrderMinRays &&
                       count < (int64_t{1} << 32);
    cudaError_t err = cudaSuccess;
    const bool timed = a->timing && reorder;
    if (timed) err = cudaEventRecord(a->ev[0], stream);
    if (order && err == cudaSuccess) {
        const int bits = RayOrderBits(count, a->order_bits);
        err = EnsureOrderScratch(a, count, bits);
        if (err != cudaSuccess) return CudaFail(err, "ray order scratch");
        err = OrderRays(args.rays, count, a->params, a->order_mode, bits, a->order_length, a->order, stream,
                        a->sm_count);
        if (err != cudaSuccess) return CudaFail(err, "ray order");
        args.order = a->order.order;
    }
    if (timed && err == cudaSuccess) err = cudaEventRecord(a->ev[1], stream);
    if (err == cudaSuccess) err = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), stream);
    if (err != cudaSuccess) return CudaFail(err, "trace counter reset");
    err = LaunchTrace(args, any, stats, shape >= 0 ? shape : a->trace_shape[any ? 1 : 0], stream, a->sm_count);
    if (err != cudaSuccess) return CudaFail(err, "trace launch");
    if (timed) {
        err = cudaEventRecord(a->ev[2], stream);
        if (err != cudaSuccess) return CudaFail(err, "trace timing event");
        a->timed_order = order;
    }
    return Ok();
}

}  // namespace

AccelParams AccelParamsOf(const yrc_accel* a) { return a->params; }
int TraceShapeOf(const yrc_accel* a, int any_hit) { return a->trace_shape[any_hit ? 1 : 0]; }
int* AccelErrorWord(yrc_accel* a) { return a->d_error; }

yrc_status CheckDeviceError(yrc_accel* a) {
    int status = 0;
    cudaError_t err = cudaMemcpy(&status, a->d_error, sizeof(int), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return CudaFail(err, "reading the device status word");
    if (status != 0) {
        cudaMemset(a->d_error, 0, sizeof(int));
        if (status & kTraceErrorStackOverflow) return Fail(YRC_ERR_DEVICE_FAULT, "traversal stack overflow");
        return Fail(YRC_ERR_DEVICE_FAULT, "device status word " + std::to_string(status));
    }
    return Ok();
}

}  // namespace yrc

// Fixed scratch of yrc_trace_stats_device_noalloc, resident on every GPU that
// loads this library until the process exits. Bytes [0, 256) hold the
// persistent-warp ray-refill counter, which must be zero when a launch starts
// (reset with cudaMemsetAsync on the caller's stream before every launch);
// from byte 256 on, the hit records (16 B per ray) or occlusion bytes (1 B per
// ray) that the stats traversal writes and nobody reads — they need no
// clearing. Host code sees this name only as a host-side stand-in: the device
// address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char yrc_noalloc_stats_scratch[256 + 16 * YRC_NOALLOC_STATS_MAX_RAYS];

namespace yrc {
namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_scratch[kNoAllocMaxDevices] = {};

// Device address of yrc_noalloc_stats_scratch on `device`, which must be the
// current device. Looked up on the first call per device and cached.
yrc_status NoAllocScratch(int device, unsigned char** out) {
    if (device < 0 || device >= kNoAllocMaxDevices) {
        return Fail(YRC_ERR_UNSUPPORTED, "yrc_trace_stats_device_noalloc: device index " + std::to_string(device) +
                                             " is beyond the " + std::to_string(kNoAllocMaxDevices) +
                                             " devices this entry point keeps scratch addresses for");
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_scratch[device]) {
        void* p = nullptr;
        const cudaError_t err = cudaGetSymbolAddress(&p, yrc_noalloc_stats_scratch);
        if (err != cudaSuccess) return CudaFail(err, "yrc_trace_stats_device_noalloc: scratch address lookup");
        g_noalloc_scratch[device] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_scratch[device];
    return Ok();
}

// Called when an accelerator is created on its device (current): looks up
// the scratch address there and loads the statistics kernels that
// yrc_trace_stats_device_noalloc launches for this accelerator. With lazy
// module loading (the CUDA 12 default) a module is loaded, and a kernel's
// code placed in device memory, only when first used; this file has no
// kernels, so the module that holds the scratch array is loaded only by the
// address lookup. Doing both at creation, which allocates anyway, leaves
// nothing for the first no-allocation call to allocate. A failure here is
// not the creation's: the no-allocation call retries the lookup and reports.
void ResolveNoAllocScratch(const yrc_accel* a) {
    unsigned char* ignored = nullptr;
    const bool looked_up = NoAllocScratch(a->device, &ignored) == YRC_OK;
    const bool loaded = PreloadStatsKernels(a->params.two_level != 0, a->params.stack_limit) == cudaSuccess;
    if (!looked_up || !loaded) cudaGetLastError();
    Ok();
}

}  // namespace
}  // namespace yrc

extern "C" {

yrc_status yrc_accel_create_flat(const yrc_geometry* geometry, const yrc_bvh_view* bvh, yrc_accel** out) {
    using namespace yrc;
    if (!out) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_create_flat: null output");
    *out = nullptr;
    std::string error;
    if (!CheckGeometry(geometry, error) || !CheckBvh(bvh, error)) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_create_flat: " + error);
    }
    Layout layout;
    int32_t root = kAbsentRef, depth = 0;
    float lo[3], hi[3];
    try {
        auto slot = [&](int64_t s) { return TriangleOrSphereRecord(*geometry, *bvh, s); };
        if (!AddBvh(bvh->nodes, bvh->node_count, slot, layout, root, lo, hi, depth, error)) {
            return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_create_flat: " + error);
        }
    } catch (const std::bad_alloc&) {
        return Fail(YRC_ERR_OUT_OF_MEMORY, "yrc_accel_create_flat: host allocation failed");
    }
    const yrc_status st = Finalize(layout, root, lo, hi, 0, depth, out);
    if (st != YRC_OK) return st;
    ResolveNoAllocScratch(*out);
    // A four-wide copy is allowed for triangle-only BVHs: their closest hit
    // does not depend on the visiting order (ties go to the smaller flat
    // index), while a sphere tie goes to the first visited.
    bool triangles_only = true;
    for (int64_t i = 0; i < bvh->primitive_count; ++i) triangles_only = triangles_only && bvh->primitives[i].kind == 0;
    (*out)->triangles_only = triangles_only;
    return st;
}

yrc_status yrc_accel_create_two_level(const yrc_geometry* geometry, const yrc_two_level_view* tl, yrc_accel** out) {
    using namespace yrc;
    if (!out) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_create_two_level: null output");
    *out = nullptr;
    std::string error;
    if (!CheckGeometry(geometry, error)) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_create_two_level: " + error);
    if (!tl || tl->blas_count < 0 || tl->instance_count < 0 || (tl->blas_count > 0 && !tl->blases) ||
        (tl->instance_count > 0 && !tl->instances) || (tl->tlas_node_count > 0 && !tl->tlas_nodes) ||
        (tl->tlas_primitive_index_count > 0 && !tl->tlas_primitive_indices) ||
        (tl->tlas_primitive_count > 0 && !tl->tlas_primitives)) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_create_two_level: invalid two-level view");
    }
    Layout layout;
    int32_t tlas_root = kAbsentRef, tlas_depth = 0;
    float lo[3], hi[3];
    try {
        // BLASes first so their refs are known when instances are written.
        std::vector<int32_t> blas_root(static_cast<size_t>(tl->blas_count), kAbsentRef);
        std::vector<std::array<float, 6>> blas_box(static_cast<size_t>(tl->blas_count));
        int32_t blas_depth = 0;
        for (int32_t b = 0; b < tl->blas_count; ++b) {
            const yrc_bvh_view& v = tl->blases[b].bvh;
            if (!CheckBvh(&v, error)) return Fail(YRC_ERR_INVALID_ARGUMENT, "BLAS " + std::to_string(b) + ": " + error);
            auto slot = [&](int64_t s) { return TriangleOrSphereRecord(*geometry, v, s); };
            float blo[3], bhi[3];
            int32_t d = 0;
            if (!AddBvh(v.nodes, v.node_count, slot, layout, blas_root[b], blo, bhi, d, error)) {
                return Fail(YRC_ERR_INVALID_ARGUMENT, "BLAS " + std::to_string(b) + ": " + error);
            }
            blas_depth = std::max(blas_depth, d);
            blas_box[b] = {blo[0], blo[1], blo[2], bhi[0], bhi[1], bhi[2]};
        }
        layout.instances.resize(static_cast<size_t>(tl->instance_count));
        for (int32_t i = 0; i < tl->instance_count; ++i) {
            const yrc_prepared_instance& src = tl->instances[i];
            Instance& dst = layout.instances[static_cast<size_t>(i)];
            const float* m = src.world_to_object;
            dst.row0 = make_float4(m[0], m[4], m[8], m[12]);
            dst.row1 = make_float4(m[1], m[5], m[9], m[13]);
            dst.row2 = make_float4(m[2], m[6], m[10], m[14]);
            const bool valid = src.blas_index >= 0 && src.blas_index < tl->blas_count;
            const std::array<float, 6> box = valid ? blas_box[src.blas_index] : std::array<float, 6>{};
            dst.box_a = make_float4(box[0], box[1], box[2], box[3]);
            dst.box_b = make_float4(box[4], box[5], IntBits(valid ? blas_root[src.blas_index] : kAbsentRef),
                                    0.0f);
        }
        auto tlas_slot = [&](int64_t s) -> Record {
            if (s < 0 || s >= tl->tlas_primitive_index_count) return SkipRecord(kRecSkip);
            const int32_t pi = tl->tlas_primitive_indices[s];
            if (pi < 0 || pi >= tl->tlas_primitive_count) return SkipRecord(kRecSkip);
            const yrc_tlas_primitive& p = tl->tlas_primitives[pi];
            if (p.kind == 1) return SphereRecord(*geometry, p.sphere);
            if (p.instance < 0 || p.instance >= tl->instance_count) return SkipRecord(kRecSkip);
            const int32_t b = tl->instances[p.instance].blas_index;
            if (b < 0 || b >= tl->blas_count) return SkipRecord(kRecSkip);
            Record r{};
            r.v0 = make_float4(0.0f, 0.0f, 0.0f, IntBits(p.instance));
            r.v1 = make_float4(0.0f, 0.0f, 0.0f, IntBits(kRecInstance << 1));
            return r;
        };
        if (!AddBvh(tl->tlas_nodes, tl->tlas_node_count, tlas_slot, layout, tlas_root, lo, hi, tlas_depth, error)) {
            return Fail(YRC_ERR_INVALID_ARGUMENT, "TLAS: " + error);
        }
        tlas_depth += blas_depth;
    } catch (const std::bad_alloc&) {
        return Fail(YRC_ERR_OUT_OF_MEMORY, "yrc_accel_create_two_level: host allocation failed");
    }
    const yrc_status st = Finalize(layout, tlas_root, lo, hi, 1, tlas_depth, out);
    if (st == YRC_OK) ResolveNoAllocScratch(*out);
    return st;
}

void yrc_accel_destroy(yrc_accel* accel) { yrc::FreeAccel(accel); }

int64_t yrc_accel_device_bytes(const yrc_accel* accel) { return accel ? accel->device_bytes : 0; }

yrc_status yrc_trace_device(yrc_accel* accel, const yrc_ray* rays, int64_t count, int32_t flags, yrc_hit* hits,
                            int32_t* instances, uint8_t* occluded, void* stream) {
    using namespace yrc;
    if (!accel || count < 0 || (count > 0 && !rays)) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_trace_device: bad argument");
    const bool any = (flags & YRC_TRACE_ANY) != 0;
    if (count > 0 && ((any && !occluded) || (!any && !hits))) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_trace_device: missing output buffer");
    }
    std::lock_guard<std::mutex> lock(accel->mutex);
    cudaSetDevice(accel->device);
    return LaunchInternal(accel, rays, count, flags & ~YRC_TRACE_STATS, hits, instances, occluded, nullptr, nullptr,
                          nullptr, accel->d_counter, static_cast<cudaStream_t>(stream), true);
}

yrc_status yrc_trace_stats_device(yrc_accel* accel, const yrc_ray* rays, int64_t count, int32_t flags,
                                  uint32_t* node_tests, uint32_t* triangle_tests, uint32_t* sphere_tests,
                                  void* stream) {
    using namespace yrc;
    if (!accel || count < 0 || (count > 0 && !rays)) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_trace_stats_device: bad argument");
    }
    std::lock_guard<std::mutex> lock(accel->mutex);
    cudaSetDevice(accel->device);
    const bool any = (flags & YRC_TRACE_ANY) != 0;
    // The stats kernel still writes its primary output; route it to scratch.
    void* scratch = nullptr;
    cudaError_t err = cudaMallocAsync(&scratch, static_cast<size_t>(std::max<int64_t>(count, 1)) * (any ? 1 : 16),
                                      static_cast<cudaStream_t>(stream));
    if (err != cudaSuccess) return CudaFail(err, "stats scratch");
    yrc_status s = LaunchInternal(accel, rays, count, flags | YRC_TRACE_STATS, any ? nullptr : static_cast<yrc_hit*>(scratch),
                                  nullptr, any ? static_cast<uint8_t*>(scratch) : nullptr, node_tests, triangle_tests,
                                  sphere_tests, accel->d_counter, static_cast<cudaStream_t>(stream));
    cudaFreeAsync(scratch, static_cast<cudaStream_t>(stream));
    return s;
}

yrc_status yrc_trace_stats_device_noalloc(yrc_accel* accel, const yrc_ray* rays, int64_t count, int32_t flags,
                                          uint32_t* node_tests, uint32_t* triangle_tests, uint32_t* sphere_tests,
                                          void* stream) {
    using namespace yrc;
    if (!accel || count < 0 || (count > 0 && !rays)) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_trace_stats_device_noalloc: bad argument");
    }
    if (count > YRC_NOALLOC_STATS_MAX_RAYS) {
        return Fail(YRC_ERR_INVALID_ARGUMENT,
                    "yrc_trace_stats_device_noalloc: " + std::to_string(count) + " rays exceed the fixed maximum of " +
                        std::to_string(YRC_NOALLOC_STATS_MAX_RAYS) +
                        " per call (the size of its preallocated scratch); split the batch or use "
                        "yrc_trace_stats_device");
    }
    std::lock_guard<std::mutex> lock(accel->mutex);
    cudaSetDevice(accel->device);
    unsigned char* scratch = nullptr;
    const yrc_status set_up = NoAllocScratch(accel->device, &scratch);
    if (set_up != YRC_OK) return set_up;
    const bool any = (flags & YRC_TRACE_ANY) != 0;
    // LaunchInternal zeroes the counter (cudaMemsetAsync) before the launch.
    auto* counter = reinterpret_cast<unsigned long long*>(scratch);
    unsigned char* discard = scratch + 256;
    return LaunchInternal(accel, rays, count, flags | YRC_TRACE_STATS, any ? nullptr : reinterpret_cast<yrc_hit*>(discard),
                          nullptr, any ? discard : nullptr, node_tests, triangle_tests, sphere_tests, counter,
                          static_cast<cudaStream_t>(stream));
}

yrc_status yrc_trace_host(yrc_accel* accel, const yrc_ray* rays, int64_t count, int32_t flags, yrc_hit* hits,
                          int32_t* instances, uint8_t* occluded, yrc_trace_stats* stats) {
    using namespace yrc;
    if (!accel || count < 0 || (count > 0 && !rays)) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_trace_host: bad argument");
    const bool any = (flags & YRC_TRACE_ANY) != 0;
    const bool want_stats = (flags & YRC_TRACE_STATS) != 0 && stats != nullptr;
    if (count > 0 && ((any && !occluded) || (!any && !hits))) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_trace_host: missing output buffer");
    }
    std::lock_guard<std::mutex> lock(accel->mutex);
    cudaSetDevice(accel->device);
    HostPipeline& p = accel->pipe;
    cudaError_t err = cudaSuccess;
    if (p.chunk == 0) {
        // 512K rays (16 MiB of rays) per chunk: enough chunks in a large
        // batch that the copies of one overlap the traversal of another and
        // only one chunk's upload and readback are exposed.
        p.chunk = int64_t{1} << 19;
        err = cudaMalloc(reinterpret_cast<void**>(&p.d_counters), sizeof(unsigned long long) * HostPipeline::kStreams);
        for (int s = 0; s < HostPipeline::kStreams && err == cudaSuccess; ++s) {
            err = cudaStreamCreateWithFlags(&p.streams[s], cudaStreamNonBlocking);
            if (err == cudaSuccess) err = cudaMalloc(&p.d_rays[s], static_cast<size_t>(p.chunk) * sizeof(yrc_ray));
            if (err == cudaSuccess) err = cudaMalloc(&p.d_out[s], static_cast<size_t>(p.chunk) * sizeof(yrc_hit));
            if (err == cudaSuccess)
                err = cudaMalloc(reinterpret_cast<void**>(&p.d_inst[s]), static_cast<size_t>(p.chunk) * sizeof(int32_t));
            if (err == cudaSuccess)
                err = cudaMalloc(reinterpret_cast<void**>(&p.d_stats[s]), static_cast<size_t>(p.chunk) * 3 * sizeof(uint32_t));
        }
        if (err != cudaSuccess) {
            p.chunk = 0;
            return CudaFail(err, "yrc_trace_host pipeline setup");
        }
    }
    std::vector<uint32_t> host_stats;
    if (want_stats) host_stats.resize(static_cast<size_t>(std::min(count, p.chunk)) * 3);
    yrc_trace_stats total{0, 0, 0, static_cast<uint64_t>(count)};
    int64_t done = 0;
    int chunk_id = 0;
    while (done < count && err == cudaSuccess) {
        const int s = chunk_id % HostPipeline::kStreams;
        const int64_t n = std::min(p.chunk, count - done);
        cudaStream_t st = p.streams[s];
        if (want_stats) err = cudaStreamSynchronize(st);  // host_stats buffer is reused per chunk
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(p.d_rays[s], rays + done, static_cast<size_t>(n) * sizeof(yrc_ray),
                                  cudaMemcpyHostToDevice, st);
        if (err != cudaSuccess) break;
        uint32_t* ds = p.d_stats[s];
        yrc_status ls = LaunchInternal(accel, static_cast<const yrc_ray*>(p.d_rays[s]), n,
                                       want_stats ? flags : (flags & ~YRC_TRACE_STATS),
                                       any ? nullptr : static_cast<yrc_hit*>(p.d_out[s]), instances ? p.d_inst[s] : nullptr,
                                       any ? static_cast<uint8_t*>(p.d_out[s]) : nullptr, want_stats ? ds : nullptr,
                                       want_stats ? ds + n : nullptr, want_stats ? ds + 2 * n : nullptr,
                                       p.d_counters + s, st, false, accel->host_shape[any ? 1 : 0].load());
        if (ls != YRC_OK) return ls;
        if (any) {
            err = cudaMemcpyAsync(occluded + done, p.d_out[s], static_cast<size_t>(n), cudaMemcpyDeviceToHost, st);
        } else {
            err = cudaMemcpyAsync(hits + done, p.d_out[s], static_cast<size_t>(n) * sizeof(yrc_hit),
                                  cudaMemcpyDeviceToHost, st);
            if (err == cudaSuccess && instances)
                err = cudaMemcpyAsync(instances + done, p.d_inst[s], static_cast<size_t>(n) * sizeof(int32_t),
                                      cudaMemcpyDeviceToHost, st);
        }
        if (want_stats && err == cudaSuccess) {
            err = cudaMemcpyAsync(host_stats.data(), ds, static_cast<size_t>(n) * 3 * sizeof(uint32_t),
                                  cudaMemcpyDeviceToHost, st);
            if (err == cudaSuccess) err = cudaStreamSynchronize(st);
            for (int64_t i = 0; i < n && err == cudaSuccess; ++i) {
                total.node_tests += host_stats[static_cast<size_t>(i)];
                total.triangle_tests += host_stats[static_cast<size_t>(n + i)];
                total.sphere_tests += host_stats[static_cast<size_t>(2 * n + i)];
            }
        }
        done += n;
        ++chunk_id;
    }
    for (int s = 0; s < HostPipeline::kStreams; ++s) {
        const cudaError_t e2 = cudaStreamSynchronize(p.streams[s]);
        if (err == cudaSuccess) err = e2;
    }
    if (err != cudaSuccess) return CudaFail(err, "yrc_trace_host");
    if (want_stats) *stats = total;
    return CheckDeviceError(accel);
}

yrc_status yrc_probe_device(yrc_accel* accel, const yrc_ray* rays, const yrc_probe_target* targets, int64_t count,
                            yrc_hit* hits, int32_t* instances, int32_t* counts, uint8_t* exhausted, void* stream) {
    using namespace yrc;
    if (!accel || count < 0 || (count > 0 && (!rays || !targets || !hits || !counts || !exhausted))) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_probe_device: bad argument");
    }
    if (count == 0) return Ok();
    std::lock_guard<std::mutex> lock(accel->mutex);
    cudaSetDevice(accel->device);
    ProbeArgs args{};
    args.accel = accel->params;
    args.rays = reinterpret_cast<const float4*>(rays);
    args.targets = targets;
    args.count = count;
    args.hits = hits;
    args.instances = instances;
    args.counts = counts;
    args.exhausted = exhausted;
    args.error = accel->d_error;
    const cudaError_t err = LaunchProbe(args, static_cast<cudaStream_t>(stream), accel->sm_count);
    if (err != cudaSuccess) return CudaFail(err, "probe launch");
    return Ok();
}

yrc_status yrc_accel_set_trace_shape(yrc_accel* accel, int32_t any_hit, int32_t shape) {
    if (!accel || shape < 0 || shape >= yrc::kTraceShapes) {
        return yrc::Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_set_trace_shape: bad argument");
    }
    accel->trace_shape[any_hit ? 1 : 0] = shape;
    return yrc::Ok();
}

yrc_status yrc_accel_set_host_trace_shape(yrc_accel* accel, int32_t any_hit, int32_t shape) {
    if (!accel || shape < -1 || shape >= yrc::kTraceShapes) {
        return yrc::Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_set_host_trace_shape: bad argument");
    }
    accel->host_shape[any_hit ? 1 : 0] = shape;
    return yrc::Ok();
}

int32_t yrc_accel_get_host_trace_shape(const yrc_accel* accel, int32_t any_hit) {
    return accel ? accel->host_shape[any_hit ? 1 : 0].load() : -2;
}

yrc_status yrc_accel_autotune_host(yrc_accel* accel, const yrc_ray* rays, int64_t count, int32_t flags,
                                   float* times_ms) {
    using namespace yrc;
    if (!accel || count <= 0 || !rays) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_autotune_host: bad argument");
    const bool any = (flags & YRC_TRACE_ANY) != 0;
    const int32_t trace_flags = flags & YRC_TRACE_ANY;
    // Pinned output, as a caller that cares about this path's speed has.
    uint8_t* out = nullptr;
    cudaSetDevice(accel->device);
    const cudaError_t aerr = cudaMallocHost(reinterpret_cast<void**>(&out),
                                            static_cast<size_t>(count) * (any ? 1 : sizeof(yrc_hit)));
    if (aerr != cudaSuccess) return CudaFail(aerr, "yrc_accel_autotune_host output");
    float totals[kTraceShapes] = {};
    const int saved = accel->host_shape[any ? 1 : 0].load();
    yrc_status status = Ok();
    for (int shape = 0; shape < kTraceShapes && status == YRC_OK; ++shape) {
        accel->host_shape[any ? 1 : 0] = shape;
        double total = 0.0;
        for (int rep = 0; rep < 3 && status == YRC_OK; ++rep) {  // first repetition warms up
            const auto t0 = std::chrono::steady_clock::now();
            status = yrc_trace_host(accel, rays, count, trace_flags, any ? nullptr : reinterpret_cast<yrc_hit*>(out),
                                    nullptr, any ? out : nullptr, nullptr);
            const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            if (rep > 0) total += ms;
        }
        totals[shape] = static_cast<float>(total);
        if (times_ms) times_ms[shape] = static_cast<float>(total / 2.0);
    }
    cudaFreeHost(out);
    if (status != YRC_OK) {
        accel->host_shape[any ? 1 : 0] = saved;
        return status;
    }
    // As the device autotuner: the lowest-index shape within 2 % of the fastest.
    float best = totals[0];
    for (int shape = 1; shape < kTraceShapes; ++shape) best = totals[shape] < best ? totals[shape] : best;
    int best_shape = 0;
    while (best_shape + 1 < kTraceShapes && totals[best_shape] > 1.02f * best) ++best_shape;
    accel->host_shape[any ? 1 : 0] = best_shape;
    return Ok();
}

int32_t yrc_accel_get_trace_shape(const yrc_accel* accel, int32_t any_hit) {
    return accel ? accel->trace_shape[any_hit ? 1 : 0] : -1;
}

yrc_status yrc_accel_set_wide(yrc_accel* accel, int32_t enable) {
    using namespace yrc;
    if (!accel) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_set_wide: null accelerator");
    std::lock_guard<std::mutex> lock(accel->mutex);
    if (enable && !accel->d_wide) {
        if (!accel->triangles_only || accel->params.two_level || accel->params.root_ref < 0) {
            return Fail(YRC_ERR_UNSUPPORTED, "yrc_accel_set_wide: no four-wide copy (two-level BVH, spheres or a leaf root)");
        }
        cudaSetDevice(accel->device);
        std::vector<NodePair> pairs(static_cast<size_t>(accel->pair_count));
        cudaError_t err = cudaMemcpy(pairs.data(), accel->d_pairs, sizeof(NodePair) * pairs.size(), cudaMemcpyDeviceToHost);
        if (err != cudaSuccess) return CudaFail(err, "yrc_accel_set_wide: reading the binary nodes");
        WideLayout w;
        BuildWide(pairs, accel->params.root_ref, w);
        if (w.nodes.empty() || w.stack > kMaxTraceStack) {
            return Fail(YRC_ERR_UNSUPPORTED, "yrc_accel_set_wide: four-wide hierarchy too deep");
        }
        err = Upload(&accel->d_wide, w.nodes, accel->device_bytes);
        if (err != cudaSuccess) {
            cudaFree(accel->d_wide);
            accel->d_wide = nullptr;
            return CudaFail(err, "yrc_accel_set_wide: upload");
        }
        accel->params.wide_root = w.root;
        accel->params.wide_stack_limit = w.stack;
    }
    accel->wide_enabled = enable != 0;
    accel->params.wide = accel->wide_enabled ? accel->d_wide : nullptr;
    return yrc::Ok();
}

int32_t yrc_accel_get_wide(const yrc_accel* accel) { return accel && accel->wide_enabled ? 1 : 0; }

yrc_status yrc_accel_set_ray_order(yrc_accel* accel, int32_t mode, int32_t key_bits, float length) {
    using namespace yrc;
    if (!accel || mode < YRC_RAY_ORDER_OFF || mode > YRC_RAY_ORDER_TWO_POINT || key_bits < 0 ||
        key_bits > kRayOrderMaxBits || !(length >= 0.0f) || !(length <= 16.0f)) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_set_ray_order: bad argument");
    }
    std::lock_guard<std::mutex> lock(accel->mutex);
    accel->order_mode = mode;
    accel->order_bits = key_bits;
    accel->order_length = length;
    return Ok();
}

int32_t yrc_accel_get_ray_order(const yrc_accel* accel) { return accel ? accel->order_mode : -1; }

yrc_status yrc_accel_set_timing(yrc_accel* accel, int32_t enable) {
    using namespace yrc;
    if (!accel) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_set_timing: null accelerator");
    std::lock_guard<std::mutex> lock(accel->mutex);
    cudaSetDevice(accel->device);
    if (enable && !accel->ev[0]) {
        for (cudaEvent_t& e : accel->ev) {
            const cudaError_t err = cudaEventCreate(&e);
            if (err != cudaSuccess) return CudaFail(err, "yrc_accel_set_timing");
        }
    }
    accel->timing = enable != 0;
    return Ok();
}

yrc_status yrc_accel_last_timing(yrc_accel* accel, float* order_ms, float* trace_ms) {
    using namespace yrc;
    if (!accel || !order_ms || !trace_ms) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_last_timing: bad argument");
    std::lock_guard<std::mutex> lock(accel->mutex);
    if (!accel->timing) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_last_timing: timing is off");
    cudaSetDevice(accel->device);
    cudaError_t err = cudaEventSynchronize(accel->ev[2]);
    if (err == cudaSuccess) err = cudaEventElapsedTime(order_ms, accel->ev[0], accel->ev[1]);
    if (err == cudaSuccess) err = cudaEventElapsedTime(trace_ms, accel->ev[1], accel->ev[2]);
    if (err != cudaSuccess) return CudaFail(err, "yrc_accel_last_timing");
    if (!accel->timed_order) *order_ms = 0.0f;
    return Ok();
}

yrc_status yrc_accel_autotune(yrc_accel* accel, const yrc_ray* rays, int64_t count, int32_t flags, void* stream,
                              float* times_ms) {
    using namespace yrc;
    if (!accel || count <= 0 || !rays) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_autotune: bad argument");
    const bool any = (flags & YRC_TRACE_ANY) != 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lock(accel->mutex);
    cudaSetDevice(accel->device);
    void* out = nullptr;
    cudaError_t err = cudaMallocAsync(&out, static_cast<size_t>(count) * (any ? 1 : 16), st);
    if (err != cudaSuccess) return CudaFail(err, "autotune scratch");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float totals[kTraceShapes] = {};
    yrc_status status = Ok();
    for (int shape = 0; shape < kTraceShapes && status == YRC_OK; ++shape) {
        accel->trace_shape[any ? 1 : 0] = shape;
        float total = 0.0f;
        for (int rep = 0; rep < 3 && status == YRC_OK; ++rep) {  // first repetition warms up
            cudaEventRecord(e0, st);
            status = LaunchInternal(accel, rays, count, flags & YRC_TRACE_ANY, any ? nullptr : static_cast<yrc_hit*>(out),
                                    nullptr, any ? static_cast<uint8_t*>(out) : nullptr, nullptr, nullptr, nullptr,
                                    accel->d_counter, st, true);
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) total += ms;
        }
        if (times_ms) times_ms[shape] = total / 2.0f;
        totals[shape] = total;
    }
    // The lowest-index shape within 2 % of the fastest: the shapes often time
    // within run-to-run noise of each other, and a stable choice keeps the
    // kernel a caller tuned for (and profiled) the same from run to run.
    float best = totals[0];
    for (int shape = 1; shape < kTraceShapes; ++shape) best = totals[shape] < best ? totals[shape] : best;
    int best_shape = 0;
    while (best_shape + 1 < kTraceShapes && totals[best_shape] > 1.02f * best) ++best_shape;
    accel->trace_shape[any ? 1 : 0] = best_shape;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(out, st);
    err = cudaStreamSynchronize(st);
    if (status != YRC_OK) return status;
    if (err != cudaSuccess) return CudaFail(err, "autotune");
    return Ok();
}

yrc_status yrc_accel_check(yrc_accel* accel) {
    if (!accel) return yrc::Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_accel_check: null accelerator");
    std::lock_guard<std::mutex> lock(accel->mutex);
    cudaSetDevice(accel->device);
    const cudaError_t err = cudaDeviceSynchronize();
    if (err != cudaSuccess) return yrc::Fail(YRC_ERR_CUDA, std::string("synchronize: ") + cudaGetErrorString(err));
    return yrc::CheckDeviceError(accel);
}

yrc_status yrc_stream_synchronize(void* stream) {
    const cudaError_t err = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    if (err != cudaSuccess) return yrc::Fail(YRC_ERR_CUDA, std::string("stream synchronize: ") + cudaGetErrorString(err));
    return yrc::Ok();
}

}  // extern "C"
