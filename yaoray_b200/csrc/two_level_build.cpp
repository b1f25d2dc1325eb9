// Host-side two-level (TLAS over instances, one BLAS per mesh primitive)
// builder with the reference's TwoLevelBvh layout
// (src/accel/two_level_bvh.cpp:51-109,257-331):
//   * one BLAS per RenderPrimitive, built over that primitive alone, whose
//     RenderBvhPrimitive.mesh_primitive is rebased to the primitive's index
//     and flat_triangle_index to the running triangle count;
//   * an identity instance per primitive when the geometry has no instance
//     table, else exactly the explicit instances (checked invertible);
//   * a TLAS built over instance world boxes (the 8 transformed BLAS corners)
//     and spheres with the same SAH hierarchy builder.
// Matrix inverse and point transforms use the reference's expression order
// (src/core/transform.cpp:30-44,147-197) so that world_to_object matches bit
// for bit: the traversal kernels transform rays with it.
#include "yrc_internal.hpp"
#include "yrc_math_host.hpp"

#include <cmath>
#include <cstring>

namespace yrc {

struct HostTwoLevel {
    struct Blas {
        int32_t mesh_primitive = -1;
        Box object_bounds;
        HostBvh bvh;
    };
    std::vector<Blas> blases;
    std::vector<yrc_prepared_instance> instances;
    HostBvh tlas;  // nodes / primitive_indices / max_depth
    std::vector<yrc_tlas_primitive> tlas_primitives;
    // Views handed out by yrc_two_level_get_view.
    std::vector<yrc_blas_view> blas_views;
};

namespace {

Box TransformBox(const float m[16], const Box& b) {
    Box r;
    for (int corner = 0; corner < 8; ++corner) {
        const float p[3] = {(corner & 1) ? b.hi.x : b.lo.x, (corner & 2) ? b.hi.y : b.lo.y,
                            (corner & 4) ? b.hi.z : b.lo.z};
        float q[3];
        TransformPointRef(m, p, q);
        // Union(bounds, point): keep the accumulated value unless strictly beyond.
        r.lo = {q[0] < r.lo.x ? q[0] : r.lo.x, q[1] < r.lo.y ? q[1] : r.lo.y, q[2] < r.lo.z ? q[2] : r.lo.z};
        r.hi = {r.hi.x < q[0] ? q[0] : r.hi.x, r.hi.y < q[1] ? q[1] : r.hi.y, r.hi.z < q[2] ? q[2] : r.hi.z};
    }
    return r;
}

bool FiniteBox(const Box& b) {
    return std::isfinite(b.lo.x) && std::isfinite(b.lo.y) && std::isfinite(b.lo.z) && std::isfinite(b.hi.x) &&
           std::isfinite(b.hi.y) && std::isfinite(b.hi.z);
}

void SetBox(const Box& b, float lo[3], float hi[3]) {
    lo[0] = b.lo.x; lo[1] = b.lo.y; lo[2] = b.lo.z;
    hi[0] = b.hi.x; hi[1] = b.hi.y; hi[2] = b.hi.z;
}

Box GetBox(const float lo[3], const float hi[3]) {
    Box b;
    b.lo = {lo[0], lo[1], lo[2]};
    b.hi = {hi[0], hi[1], hi[2]};
    return b;
}

bool BuildTlas(const yrc_geometry& g, const yrc_bvh_options& options, HostTwoLevel& tl, std::string& error) {
    std::vector<BuildRef> refs;
    tl.tlas_primitives.clear();
    for (size_t i = 0; i < tl.instances.size(); ++i) {
        const yrc_prepared_instance& inst = tl.instances[i];
        const Box wb = GetBox(inst.world_bounds_min, inst.world_bounds_max);
        yrc_tlas_primitive p{};
        p.kind = 0;
        p.instance = static_cast<int32_t>(i);
        p.sphere = -1;
        SetBox(wb, p.world_bounds_min, p.world_bounds_max);
        const Vec3 c{(wb.lo.x + wb.hi.x) * 0.5f, (wb.lo.y + wb.hi.y) * 0.5f, (wb.lo.z + wb.hi.z) * 0.5f};
        refs.push_back(BuildRef{static_cast<int32_t>(tl.tlas_primitives.size()), wb, c});
        tl.tlas_primitives.push_back(p);
    }
    for (int32_t s = 0; s < g.sphere_count; ++s) {
        const yrc_sphere& sp = g.spheres[s];
        const float r = sp.radius;
        Box b;
        b.lo = {sp.center[0] - r, sp.center[1] - r, sp.center[2] - r};
        b.hi = {sp.center[0] + r, sp.center[1] + r, sp.center[2] + r};
        if (!(r > 0.0f) || !FiniteBox(b)) {
            error = "TLAS build encountered invalid sphere data";
            return false;
        }
        yrc_tlas_primitive p{};
        p.kind = 1;
        p.instance = -1;
        p.sphere = s;
        SetBox(b, p.world_bounds_min, p.world_bounds_max);
        refs.push_back(BuildRef{static_cast<int32_t>(tl.tlas_primitives.size()), b,
                                Vec3{sp.center[0], sp.center[1], sp.center[2]}});
        tl.tlas_primitives.push_back(p);
    }
    tl.tlas = HostBvh{};
    return BuildHierarchy(refs, options, tl.tlas, error);
}

bool BuildTwoLevel(const yrc_geometry& g, const yrc_bvh_options& options, HostTwoLevel& tl, std::string& error,
                   bool device = false, int32_t* device_blases = nullptr) {
    int32_t flat_offset = 0;
    for (int32_t i = 0; i < g.primitive_count; ++i) {
        yrc_geometry one = g;
        one.primitives = &g.primitives[i];
        one.primitive_count = 1;
        one.spheres = nullptr;
        one.sphere_count = 0;
        one.instances = nullptr;
        one.instance_count = 0;
        HostTwoLevel::Blas blas;
        bool on_device = false;
        if (!BuildFlatBvh(one, options, blas.bvh, error, device, &on_device)) return false;
        if (on_device && device_blases) ++*device_blases;
        if (blas.bvh.nodes.empty()) {
            error = "BLAS build encountered an empty mesh primitive";
            return false;
        }
        for (yrc_bvh_primitive& p : blas.bvh.primitives) {
            p.mesh_primitive = i;
            p.flat_triangle_index += flat_offset;
        }
        blas.mesh_primitive = i;
        blas.object_bounds = GetBox(blas.bvh.nodes[0].bounds_min, blas.bvh.nodes[0].bounds_max);
        tl.blases.push_back(std::move(blas));
        flat_offset += static_cast<int32_t>(g.primitives[i].index_count / 3);
    }

    const float identity[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    if (g.instance_count == 0) {
        for (int32_t i = 0; i < g.primitive_count; ++i) {
            yrc_prepared_instance inst{};
            inst.primitive = i;
            inst.blas_index = i;
            std::memcpy(inst.object_to_world, identity, sizeof(identity));
            std::memcpy(inst.world_to_object, identity, sizeof(identity));
            SetBox(tl.blases[static_cast<size_t>(i)].object_bounds, inst.world_bounds_min, inst.world_bounds_max);
            tl.instances.push_back(inst);
        }
    } else {
        for (int32_t k = 0; k < g.instance_count; ++k) {
            const yrc_instance& src = g.instances[k];
            const int32_t prim = src.primitive;
            if (prim < 0 || static_cast<size_t>(prim) >= tl.blases.size()) {
                error = "instance references an invalid mesh primitive";
                return false;
            }
            if (!IsInvertibleAffineRef(src.object_to_world)) {
                error = "instance transform is singular or non-finite";
                return false;
            }
            yrc_prepared_instance inst{};
            inst.primitive = prim;
            inst.blas_index = prim;
            std::memcpy(inst.object_to_world, src.object_to_world, sizeof(inst.object_to_world));
            InverseRef(src.object_to_world, inst.world_to_object);
            SetBox(TransformBox(src.object_to_world, tl.blases[static_cast<size_t>(prim)].object_bounds),
                   inst.world_bounds_min, inst.world_bounds_max);
            tl.instances.push_back(inst);
        }
    }
    return BuildTlas(g, options, tl, error);
}

}  // namespace
}  // namespace yrc

struct yrc_two_level {
    yrc::HostTwoLevel tl;
};

extern "C" {

yrc_status yrc_two_level_build(const yrc_geometry* geometry, const yrc_bvh_options* options, yrc_two_level** out) {
    if (!geometry || !out) return yrc::Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_two_level_build: null argument");
    *out = nullptr;
    yrc_bvh_options opts;
    yrc_bvh_options_default(&opts);
    if (options) opts = *options;
    auto holder = new (std::nothrow) yrc_two_level();
    if (!holder) return yrc::Fail(YRC_ERR_OUT_OF_MEMORY, "yrc_two_level_build: host allocation failed");
    std::string error;
    try {
        if (!yrc::BuildTwoLevel(*geometry, opts, holder->tl, error)) {
            delete holder;
            return yrc::Fail(YRC_ERR_BUILD, error);
        }
    } catch (const std::exception& e) {
        delete holder;
        return yrc::Fail(YRC_ERR_OUT_OF_MEMORY, std::string("yrc_two_level_build: ") + e.what());
    }
    *out = holder;
    return yrc::Ok();
}

yrc_status yrc_two_level_build_device(const yrc_geometry* geometry, const yrc_bvh_options* options,
                                      yrc_two_level** out, int32_t* device_blases) {
    if (!geometry || !out) return yrc::Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_two_level_build_device: null argument");
    *out = nullptr;
    if (device_blases) *device_blases = 0;
    yrc_bvh_options opts;
    yrc_bvh_options_default(&opts);
    if (options) opts = *options;
    auto holder = new (std::nothrow) yrc_two_level();
    if (!holder) return yrc::Fail(YRC_ERR_OUT_OF_MEMORY, "yrc_two_level_build_device: host allocation failed");
    std::string error;
    try {
        if (!yrc::BuildTwoLevel(*geometry, opts, holder->tl, error, true, device_blases)) {
            delete holder;
            return yrc::Fail(error.rfind("device BVH build", 0) == 0 ? YRC_ERR_CUDA : YRC_ERR_BUILD, error);
        }
    } catch (const std::exception& e) {
        delete holder;
        return yrc::Fail(YRC_ERR_OUT_OF_MEMORY, std::string("yrc_two_level_build_device: ") + e.what());
    }
    *out = holder;
    return yrc::Ok();
}

yrc_status yrc_two_level_get_view(const yrc_two_level* two_level, yrc_two_level_view* view) {
    if (!two_level || !view) return yrc::Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_two_level_get_view: null argument");
    auto& tl = const_cast<yrc_two_level*>(two_level)->tl;
    tl.blas_views.clear();
    for (const auto& b : tl.blases) {
        yrc_blas_view v{};
        v.mesh_primitive = b.mesh_primitive;
        v.object_bounds_min[0] = b.object_bounds.lo.x;
        v.object_bounds_min[1] = b.object_bounds.lo.y;
        v.object_bounds_min[2] = b.object_bounds.lo.z;
        v.object_bounds_max[0] = b.object_bounds.hi.x;
        v.object_bounds_max[1] = b.object_bounds.hi.y;
        v.object_bounds_max[2] = b.object_bounds.hi.z;
        v.bvh = yrc::ViewOf(b.bvh);
        tl.blas_views.push_back(v);
    }
    view->blases = tl.blas_views.data();
    view->blas_count = static_cast<int32_t>(tl.blas_views.size());
    view->instances = tl.instances.data();
    view->instance_count = static_cast<int32_t>(tl.instances.size());
    view->tlas_nodes = tl.tlas.nodes.data();
    view->tlas_node_count = static_cast<int64_t>(tl.tlas.nodes.size());
    view->tlas_primitive_indices = tl.tlas.primitive_indices.data();
    view->tlas_primitive_index_count = static_cast<int64_t>(tl.tlas.primitive_indices.size());
    view->tlas_primitives = tl.tlas_primitives.data();
    view->tlas_primitive_count = static_cast<int64_t>(tl.tlas_primitives.size());
    view->tlas_max_depth = tl.tlas.max_depth;
    return yrc::Ok();
}

void yrc_two_level_destroy(yrc_two_level* two_level) { delete two_level; }

}  // extern "C"
