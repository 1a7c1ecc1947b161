#pragma once

/// \file gwn_geometry.cuh
/// \brief Device geometry: accessor, owning object, upload and position update.
///
/// Mirrors smallgwn's include/gwn/gwn_geometry.cuh:19-149 (same accessor layout, object
/// semantics and function signatures); the work is done by gwnb_geometry_upload_f32 /
/// gwnb_geometry_update_f32 in libgwnb.so.

#include <cuda/std/span>
#include <cuda_runtime_api.h>

#include <cstddef>

#include "gwn_utils.cuh"

namespace gwn {

template <gwn_real_type Real, gwn_index_type Index = std::uint32_t> struct gwn_geometry_accessor {
    using real_type = Real;
    using index_type = Index;

    cuda::std::span<Real> vertex_x{};
    cuda::std::span<Real> vertex_y{};
    cuda::std::span<Real> vertex_z{};
    cuda::std::span<Index> tri_i0{};
    cuda::std::span<Index> tri_i1{};
    cuda::std::span<Index> tri_i2{};

    constexpr std::size_t vertex_count() const noexcept { return vertex_x.size(); }
    constexpr std::size_t triangle_count() const noexcept { return tri_i0.size(); }
    constexpr bool is_valid() const noexcept {
        return vertex_x.size() == vertex_y.size() && vertex_x.size() == vertex_z.size() &&
               tri_i0.size() == tri_i1.size() && tri_i0.size() == tri_i2.size() && gwn_span_has_storage(vertex_x) &&
               gwn_span_has_storage(vertex_y) && gwn_span_has_storage(vertex_z) && gwn_span_has_storage(tri_i0) &&
               gwn_span_has_storage(tri_i1) && gwn_span_has_storage(tri_i2);
    }
};

namespace detail {

template <gwn_real_type Real, gwn_index_type Index>
[[nodiscard]] inline gwnb_geometry_f32 to_gwnb(gwn_geometry_accessor<Real, Index> const &a) noexcept {
    gwnb_geometry_f32 g{};
    if constexpr (k_supported<Real, Index>) {
        g.vertex_x = a.vertex_x.data();
        g.vertex_y = a.vertex_y.data();
        g.vertex_z = a.vertex_z.data();
        g.vertex_count = a.vertex_x.size();
        g.tri_i0 = a.tri_i0.data();
        g.tri_i1 = a.tri_i1.data();
        g.tri_i2 = a.tri_i2.data();
        g.triangle_count = a.tri_i0.size();
    }
    return g;
}

template <gwn_real_type Real, gwn_index_type Index>
[[nodiscard]] inline gwn_geometry_accessor<Real, Index> from_gwnb(gwnb_geometry_f32 const &g) noexcept {
    gwn_geometry_accessor<Real, Index> a{};
    if constexpr (k_supported<Real, Index>) {
        a.vertex_x = cuda::std::span<Real>(g.vertex_x, g.vertex_count);
        a.vertex_y = cuda::std::span<Real>(g.vertex_y, g.vertex_count);
        a.vertex_z = cuda::std::span<Real>(g.vertex_z, g.vertex_count);
        a.tri_i0 = cuda::std::span<Index>(g.tri_i0, g.triangle_count);
        a.tri_i1 = cuda::std::span<Index>(g.tri_i1, g.triangle_count);
        a.tri_i2 = cuda::std::span<Index>(g.tri_i2, g.triangle_count);
    }
    return a;
}

} // namespace detail

template <gwn_real_type Real = float, gwn_index_type Index = std::uint32_t>
class gwn_geometry_object final : public gwn_noncopyable, public gwn_stream_mixin {
public:
    using real_type = Real;
    using index_type = Index;
    using accessor_type = gwn_geometry_accessor<Real, Index>;

    gwn_geometry_object() = default;
    gwn_geometry_object(gwn_geometry_object &&other) noexcept { swap(*this, other); }
    gwn_geometry_object &operator=(gwn_geometry_object other) noexcept {
        swap(*this, other);
        return *this;
    }
    ~gwn_geometry_object() { clear(); }

    void clear() noexcept {
        if (has_data()) {
            gwnb_geometry_f32 g = detail::to_gwnb(accessor_);
            gwnb_geometry_release_f32(&g, detail::gwnb_stream(stream()));
        }
        accessor_ = accessor_type{};
    }

    [[nodiscard]] accessor_type &accessor() noexcept { return accessor_; }
    [[nodiscard]] accessor_type const &accessor() const noexcept { return accessor_; }
    [[nodiscard]] std::size_t vertex_count() const noexcept { return accessor_.vertex_count(); }
    [[nodiscard]] std::size_t triangle_count() const noexcept { return accessor_.triangle_count(); }
    [[nodiscard]] bool has_data() const noexcept {
        return accessor_.vertex_count() != 0 || accessor_.triangle_count() != 0;
    }

    friend void swap(gwn_geometry_object &lhs, gwn_geometry_object &rhs) noexcept {
        using std::swap;
        swap(lhs.accessor_, rhs.accessor_);
        swap(static_cast<gwn_stream_mixin &>(lhs), static_cast<gwn_stream_mixin &>(rhs));
    }

private:
    accessor_type accessor_{};
};

/// Upload host geometry and validate indices; replaces \p object only on success.
template <gwn_real_type Real, gwn_index_type Index>
[[nodiscard]] gwn_status gwn_upload_geometry(
    gwn_geometry_object<Real, Index> &object, gwn_host_span<Real const> const x, gwn_host_span<Real const> const y,
    gwn_host_span<Real const> const z, gwn_host_span<Index const> const i0, gwn_host_span<Index const> const i1,
    gwn_host_span<Index const> const i2, cudaStream_t stream = gwn_default_stream()
) noexcept {
    if constexpr (!detail::k_supported<Real, Index>) {
        return detail::unsupported_instantiation();
    } else {
        if (x.size() != y.size() || x.size() != z.size())
            return gwn_status::invalid_argument("Vertex SoA spans must have identical lengths.");
        if (i0.size() != i1.size() || i0.size() != i2.size())
            return gwn_status::invalid_argument("Triangle SoA spans must have identical lengths.");
        gwnb_geometry_f32 staging{};
        int const rc = gwnb_geometry_upload_f32(&staging, x.data(), y.data(), z.data(), x.size(), i0.data(), i1.data(),
                                                i2.data(), i0.size(), detail::gwnb_stream(stream));
        if (rc != GWNB_OK)
            return detail::gwnb_to_status(rc);
        gwn_geometry_object<Real, Index> replacement;
        replacement.accessor() = detail::from_gwnb<Real, Index>(staging);
        replacement.set_stream(stream);
        swap(object, replacement);
        return gwn_status::ok();
    }
}

/// Enqueue host-to-device position copies (asynchronous; host memory must outlive the copy).
template <gwn_real_type Real, gwn_index_type Index>
[[nodiscard]] gwn_status gwn_update_geometry(
    gwn_geometry_object<Real, Index> &object, gwn_host_span<Real const> const x, gwn_host_span<Real const> const y,
    gwn_host_span<Real const> const z, cudaStream_t stream = gwn_default_stream()
) noexcept {
    if constexpr (!detail::k_supported<Real, Index>) {
        return detail::unsupported_instantiation();
    } else {
        if (x.size() != y.size() || x.size() != z.size())
            return gwn_status::invalid_argument("Vertex SoA spans must have identical lengths.");
        gwnb_geometry_f32 g = detail::to_gwnb(object.accessor());
        int const rc = gwnb_geometry_update_f32(&g, x.data(), y.data(), z.data(), x.size(), detail::gwnb_stream(stream));
        if (rc == GWNB_OK)
            object.set_stream(stream);
        return detail::gwnb_to_status(rc);
    }
}

} // namespace gwn
