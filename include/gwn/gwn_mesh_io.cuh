#pragma once

/// \file gwn_mesh_io.cuh
/// \brief PLY meshes and scene files for the drop-in API.
///
/// gwn_host_mesh has the fields of smallgwn's test mesh (tests/test_mesh_io.hpp:13-20) and
/// gwn_load_ply_mesh replaces its libigl loader (tests/test_mesh_io.cpp:43-92). Scene files have
/// no smallgwn counterpart: they keep geometry, a built BVH and its moments so that a later process
/// skips the build; loading refits the saved moment orders from the loaded BVH and checks them
/// equal to the saved ones.

#include <cstdint>
#include <cstdlib>
#include <filesystem>
#include <optional>
#include <string>
#include <vector>

#include "gwn_bvh.cuh"
#include "gwn_geometry.cuh"

namespace gwn {

struct gwn_host_mesh {
    std::vector<float> vertex_x;
    std::vector<float> vertex_y;
    std::vector<float> vertex_z;
    std::vector<std::uint32_t> tri_i0;
    std::vector<std::uint32_t> tri_i1;
    std::vector<std::uint32_t> tri_i2;
};

/// Reads an ASCII or binary PLY (polygons split into triangle fans) into \p mesh.
[[nodiscard]] inline gwn_status gwn_read_ply_mesh(std::filesystem::path const &path, gwn_host_mesh &mesh) noexcept try {
    gwnb_host_mesh_f32 raw{};
    int const rc = gwnb_mesh_read_ply(path.string().c_str(), &raw);
    if (rc != GWNB_OK)
        return detail::gwnb_to_status(rc);
    gwn_host_mesh out;
    out.vertex_x.assign(raw.x, raw.x + raw.vertex_count);
    out.vertex_y.assign(raw.y, raw.y + raw.vertex_count);
    out.vertex_z.assign(raw.z, raw.z + raw.vertex_count);
    out.tri_i0.assign(raw.i0, raw.i0 + raw.triangle_count);
    out.tri_i1.assign(raw.i1, raw.i1 + raw.triangle_count);
    out.tri_i2.assign(raw.i2, raw.i2 + raw.triangle_count);
    gwnb_host_mesh_free(&raw);
    mesh = std::move(out);
    return gwn_status::ok();
} catch (...) {
    return gwn_status::internal_error("Host allocation failed in gwn_read_ply_mesh.");
}

/// smallgwn's test-loader shape: the mesh, or nothing when the file cannot be read.
[[nodiscard]] inline std::optional<gwn_host_mesh> gwn_load_ply_mesh(std::filesystem::path const &path) {
    gwn_host_mesh mesh;
    if (!gwn_read_ply_mesh(path, mesh).is_ok())
        return std::nullopt;
    return mesh;
}

/// Writes \p mesh as PLY (binary little-endian, or ASCII with binary = false).
[[nodiscard]] inline gwn_status gwn_write_ply_mesh(std::filesystem::path const &path, gwn_host_mesh const &mesh,
                                                   bool const binary = true) noexcept {
    if (mesh.vertex_y.size() != mesh.vertex_x.size() || mesh.vertex_z.size() != mesh.vertex_x.size())
        return gwn_status::invalid_argument("Vertex SoA spans must have identical lengths.");
    if (mesh.tri_i1.size() != mesh.tri_i0.size() || mesh.tri_i2.size() != mesh.tri_i0.size())
        return gwn_status::invalid_argument("Triangle SoA spans must have identical lengths.");
    gwnb_host_mesh_f32 raw{};
    raw.x = const_cast<float *>(mesh.vertex_x.data());
    raw.y = const_cast<float *>(mesh.vertex_y.data());
    raw.z = const_cast<float *>(mesh.vertex_z.data());
    raw.vertex_count = mesh.vertex_x.size();
    raw.i0 = const_cast<std::uint32_t *>(mesh.tri_i0.data());
    raw.i1 = const_cast<std::uint32_t *>(mesh.tri_i1.data());
    raw.i2 = const_cast<std::uint32_t *>(mesh.tri_i2.data());
    raw.triangle_count = mesh.tri_i0.size();
    return detail::gwnb_to_status(gwnb_mesh_write_ply(path.string().c_str(), &raw, binary ? 1 : 0));
}

/// Uploads a host mesh (gwn_upload_geometry on its spans).
[[nodiscard]] inline gwn_status gwn_upload_geometry(gwn_geometry_object<float, std::uint32_t> &object,
                                                    gwn_host_mesh const &mesh,
                                                    cudaStream_t const stream = gwn_default_stream()) noexcept {
    return gwn_upload_geometry(
        object, gwn_host_span<float const>(mesh.vertex_x.data(), mesh.vertex_x.size()),
        gwn_host_span<float const>(mesh.vertex_y.data(), mesh.vertex_y.size()),
        gwn_host_span<float const>(mesh.vertex_z.data(), mesh.vertex_z.size()),
        gwn_host_span<std::uint32_t const>(mesh.tri_i0.data(), mesh.tri_i0.size()),
        gwn_host_span<std::uint32_t const>(mesh.tri_i1.data(), mesh.tri_i1.size()),
        gwn_host_span<std::uint32_t const>(mesh.tri_i2.data(), mesh.tri_i2.size()), stream);
}

/// Saves geometry, BVH and any number of moment objects of distinct orders to one file.
template <class... Moments>
[[nodiscard]] gwn_status gwn_save_scene(std::filesystem::path const &path,
                                        gwn_geometry_object<float, std::uint32_t> const &geometry,
                                        gwn_bvh4_object<float, std::uint32_t> const &bvh, Moments const &...moments) {
    static_assert(sizeof...(Moments) <= 3, "A scene holds at most one moment object per order (0, 1, 2).");
    gwnb_geometry_f32 g = detail::to_gwnb(geometry.accessor());
    auto &bvh_mut = const_cast<gwn_bvh4_object<float, std::uint32_t> &>(bvh);
    gwnb_bvh4_f32 v =
        detail::to_gwnb(bvh.accessor(), detail::object_access::aux(bvh_mut), detail::object_access::capacity(bvh_mut));
    gwnb_moment4_f32 views[3]{};
    gwnb_moment4_f32 const *ptrs[3]{};
    int count = 0;
    ((views[count] = moments.view(), ptrs[count] = &views[count], ++count), ...);
    int const rc = gwnb_scene_save_f32(path.string().c_str(), &g, &v, ptrs, count,
                                       detail::gwnb_stream(bvh.stream()));
    detail::object_access::aux(bvh_mut) = v.aux;
    return detail::gwnb_to_status(rc);
}

namespace detail {

template <int Order>
void adopt_moment(gwnb_moment4_f32 const &v, bool const present, gwn_bvh4_moment_object<Order, float, std::uint32_t> *target,
                  cudaStream_t const stream) noexcept {
    if (target == nullptr) {
        if (present) {
            gwnb_moment4_f32 tmp = v;
            gwnb_moment4_release_f32(&tmp, gwnb_stream(stream));
        }
        return;
    }
    gwn_bvh4_moment_object<Order, float, std::uint32_t> replacement;
    if (present) {
        replacement.accessor().nodes = cuda::std::span<gwn_bvh_moment_node<4, Order, float>>(
            static_cast<gwn_bvh_moment_node<4, Order, float> *>(v.nodes), v.node_count);
        replacement.accessor().bvh_revision = v.bvh_revision;
        object_access::moment_aux(replacement) = v.aux;
        replacement.set_stream(stream);
    }
    swap(*target, replacement);
}

} // namespace detail

/// Loads a scene file into new geometry and BVH objects (a fresh revision). Each non-null moment
/// pointer receives that order's moments when the file holds them and is cleared otherwise;
/// \p saved_orders (optional) receives the saved orders as bits 0-2. Replaces nothing on failure.
[[nodiscard]] inline gwn_status gwn_load_scene(std::filesystem::path const &path,
                                               gwn_geometry_object<float, std::uint32_t> &geometry,
                                               gwn_bvh4_object<float, std::uint32_t> &bvh,
                                               gwn_bvh4_moment_object<0, float, std::uint32_t> *moment0 = nullptr,
                                               gwn_bvh4_moment_object<1, float, std::uint32_t> *moment1 = nullptr,
                                               gwn_bvh4_moment_object<2, float, std::uint32_t> *moment2 = nullptr,
                                               int *saved_orders = nullptr,
                                               cudaStream_t const stream = gwn_default_stream()) noexcept {
    gwnb_geometry_f32 g{};
    gwnb_bvh4_f32 v{};
    gwnb_moment4_f32 m[3]{};
    int mask = 0;
    int const rc = gwnb_scene_load_f32(path.string().c_str(), &g, &v, m, &mask, detail::gwnb_stream(stream));
    if (rc != GWNB_OK)
        return detail::gwnb_to_status(rc);
    gwn_geometry_object<float, std::uint32_t> new_geometry;
    new_geometry.accessor() = detail::from_gwnb<float, std::uint32_t>(g);
    new_geometry.set_stream(stream);
    swap(geometry, new_geometry);
    gwn_bvh4_object<float, std::uint32_t> new_bvh;
    detail::from_gwnb(v, new_bvh.accessor());
    detail::object_access::aux(new_bvh) = v.aux;
    detail::object_access::capacity(new_bvh) = v.node_capacity;
    new_bvh.set_stream(stream);
    swap(bvh, new_bvh);
    detail::adopt_moment<0>(m[0], (mask & 1) != 0, moment0, stream);
    detail::adopt_moment<1>(m[1], (mask & 2) != 0, moment1, stream);
    detail::adopt_moment<2>(m[2], (mask & 4) != 0, moment2, stream);
    if (saved_orders != nullptr)
        *saved_orders = mask;
    return gwn_status::ok();
}

} // namespace gwn
