#pragma once

/// \file gwn_boundary.cuh
/// \brief Boundary chain of an oriented triangle mesh: accessor, owning object and builder.
///
/// Mirrors smallgwn's include/gwn/gwn_boundary.cuh:20-125 (same accessor fields and object
/// semantics): directed boundary edges with their positive net multiplicity, rows in ascending
/// (low vertex, high vertex) order. The build is gwnb_boundary_chain_build_u32 in libgwnb.so.

#include <cuda/std/span>
#include <cuda_runtime_api.h>

#include <cstddef>
#include <cstdint>

#include "gwn_geometry.cuh"
#include "gwn_utils.cuh"

namespace gwn {

template <gwn_index_type Index = std::uint32_t> struct gwn_boundary_chain_accessor {
    using index_type = Index;

    cuda::std::span<Index> start_vertex{};
    cuda::std::span<Index> end_vertex{};
    cuda::std::span<std::uint64_t> multiplicity{};
    std::size_t mesh_vertex_count{0};
    std::size_t mesh_triangle_count{0};
    bool is_built{false};

    constexpr std::size_t edge_count() const noexcept { return start_vertex.size(); }
    constexpr bool empty() const noexcept { return edge_count() == 0; }
    constexpr bool is_valid() const noexcept {
        return is_built && start_vertex.size() == end_vertex.size() && start_vertex.size() == multiplicity.size() &&
               gwn_span_has_storage(start_vertex) && gwn_span_has_storage(end_vertex) &&
               gwn_span_has_storage(multiplicity);
    }
};

namespace detail {

template <gwn_index_type Index>
[[nodiscard]] inline gwnb_boundary_chain_u32 to_gwnb(gwn_boundary_chain_accessor<Index> const &a) noexcept {
    gwnb_boundary_chain_u32 c{};
    if constexpr (std::is_same_v<Index, std::uint32_t>) {
        c.start_vertex = a.start_vertex.data();
        c.end_vertex = a.end_vertex.data();
        c.multiplicity = a.multiplicity.data();
        c.edge_count = a.start_vertex.size();
        c.mesh_vertex_count = a.mesh_vertex_count;
        c.mesh_triangle_count = a.mesh_triangle_count;
        c.is_built = a.is_built && a.is_valid() ? 1 : 0;
    }
    return c;
}

template <gwn_index_type Index>
[[nodiscard]] inline gwn_boundary_chain_accessor<Index> from_gwnb(gwnb_boundary_chain_u32 const &c) noexcept {
    gwn_boundary_chain_accessor<Index> a{};
    if constexpr (std::is_same_v<Index, std::uint32_t>) {
        a.start_vertex = cuda::std::span<Index>(c.start_vertex, c.edge_count);
        a.end_vertex = cuda::std::span<Index>(c.end_vertex, c.edge_count);
        a.multiplicity = cuda::std::span<std::uint64_t>(c.multiplicity, c.edge_count);
        a.mesh_vertex_count = c.mesh_vertex_count;
        a.mesh_triangle_count = c.mesh_triangle_count;
        a.is_built = c.is_built != 0;
    }
    return a;
}

} // namespace detail

template <gwn_index_type Index = std::uint32_t>
class gwn_boundary_chain_object final : public gwn_noncopyable, public gwn_stream_mixin {
public:
    using index_type = Index;
    using accessor_type = gwn_boundary_chain_accessor<Index>;

    gwn_boundary_chain_object() = default;
    gwn_boundary_chain_object(gwn_boundary_chain_object &&other) noexcept { swap(*this, other); }
    gwn_boundary_chain_object &operator=(gwn_boundary_chain_object other) noexcept {
        swap(*this, other);
        return *this;
    }
    ~gwn_boundary_chain_object() { clear(); }

    void clear() noexcept {
        if (accessor_.is_built) {
            gwnb_boundary_chain_u32 c = detail::to_gwnb(accessor_);
            gwnb_boundary_chain_release_u32(&c, detail::gwnb_stream(stream()));
        }
        accessor_ = accessor_type{};
    }

    [[nodiscard]] accessor_type &accessor() noexcept { return accessor_; }
    [[nodiscard]] accessor_type const &accessor() const noexcept { return accessor_; }
    [[nodiscard]] bool has_data() const noexcept { return accessor_.is_built; }

    friend void swap(gwn_boundary_chain_object &lhs, gwn_boundary_chain_object &rhs) noexcept {
        using std::swap;
        swap(lhs.accessor_, rhs.accessor_);
        swap(static_cast<gwn_stream_mixin &>(lhs), static_cast<gwn_stream_mixin &>(rhs));
    }

private:
    accessor_type accessor_{};
};

/// Build the algebraic boundary chain of \p geometry; replaces \p out only on success
/// (smallgwn include/gwn/gwn_boundary.cuh:116-125).
template <gwn_real_type Real, gwn_index_type Index>
[[nodiscard]] gwn_status gwn_build_boundary_chain(gwn_geometry_object<Real, Index> const &geometry,
                                                  gwn_boundary_chain_object<Index> &out,
                                                  cudaStream_t stream = gwn_default_stream()) noexcept {
    if constexpr (!detail::k_supported<Real, Index>) {
        return detail::unsupported_instantiation();
    } else {
        if (!geometry.accessor().is_valid())
            return gwn_status::invalid_argument("Geometry object contains no queryable data.");
        gwnb_geometry_f32 g = detail::to_gwnb(geometry.accessor());
        gwnb_boundary_chain_u32 staging{};
        int const rc = gwnb_boundary_chain_build_u32(&g, &staging, detail::gwnb_stream(stream));
        if (rc != GWNB_OK)
            return detail::gwnb_to_status(rc);
        gwn_boundary_chain_object<Index> replacement;
        replacement.accessor() = detail::from_gwnb<Index>(staging);
        replacement.set_stream(stream);
        swap(out, replacement);
        return gwn_status::ok();
    }
}

} // namespace gwn
