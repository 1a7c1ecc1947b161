#pragma once

/// \file gwn_bvh.cuh
/// \brief BVH data model: bounds, packed child references, child-AoS nodes, leaf-ordered triangle
/// records, field-SoA Taylor moment nodes, accessors and owning objects.
///
/// Layouts are identical to smallgwn's include/gwn/gwn_bvh.cuh:25-433 (the same sizes are
/// asserted below), so code that inspects or hand-assembles accessors keeps working. Owning objects
/// additionally carry the library's derived state (parent links, padded triangle records, the
/// Taylor query sidecar) as an opaque handle.

#include <cuda/std/span>

#include <cstddef>
#include <cstdint>
#include <utility>

#include "gwn_utils.cuh"

namespace gwn {

template <gwn_real_type Real> struct gwn_aabb {
    Real min_x;
    Real min_y;
    Real min_z;
    Real max_x;
    Real max_y;
    Real max_z;
};

template <gwn_real_type Real> struct gwn_bvh_triangle {
    Real v0_x{};
    Real v0_y{};
    Real v0_z{};
    Real e1_x{};
    Real e1_y{};
    Real e1_z{};
    Real e2_x{};
    Real e2_y{};
    Real e2_z{};
};

/// Bounds plus packed reference: bits 0-46 offset, bit 47 valid, bits 48-63 primitive count.
template <gwn_real_type Real> struct gwn_bvh_child {
    static constexpr int k_offset_bits = 47;
    static constexpr int k_primitive_count_bits = 16;
    static constexpr std::uint64_t k_offset_mask = (std::uint64_t(1) << k_offset_bits) - 1;
    static constexpr std::uint64_t k_valid_mask = std::uint64_t(1) << k_offset_bits;
    static constexpr int k_primitive_count_shift = k_offset_bits + 1;
    static constexpr std::uint64_t k_primitive_count_mask = (std::uint64_t(1) << k_primitive_count_bits) - 1;

    gwn_aabb<Real> bounds{};
    std::uint64_t reference = 0u;

    [[nodiscard]] static constexpr bool can_encode_offset(std::uint64_t const v) noexcept { return v <= k_offset_mask; }
    [[nodiscard]] static constexpr bool can_encode_primitive_count(std::uint64_t const v) noexcept {
        return v <= k_primitive_count_mask;
    }
    [[nodiscard]] constexpr bool is_valid() const noexcept { return (reference & k_valid_mask) != 0u; }
    [[nodiscard]] constexpr bool is_internal() const noexcept { return is_valid() && primitive_count() == 0u; }
    [[nodiscard]] constexpr bool is_leaf() const noexcept { return is_valid() && primitive_count() != 0u; }
    [[nodiscard]] constexpr std::uint64_t offset() const noexcept { return reference & k_offset_mask; }
    [[nodiscard]] constexpr std::uint32_t primitive_count() const noexcept {
        return static_cast<std::uint32_t>(reference >> k_primitive_count_shift);
    }
};

template <int Width, gwn_real_type Real> struct gwn_bvh_node {
    static_assert(Width >= 2, "BVH node width must be at least 2.");
    gwn_bvh_child<Real> children[Width]{};
    [[nodiscard]] constexpr gwn_bvh_child<Real> &child(int const slot) noexcept { return children[slot]; }
    [[nodiscard]] constexpr gwn_bvh_child<Real> const &child(int const slot) const noexcept { return children[slot]; }
};

template <gwn_real_type Real> using gwn_bvh4_node = gwn_bvh_node<4, Real>;

static_assert(sizeof(gwn_bvh_child<float>) == 32);
static_assert(sizeof(gwn_bvh_triangle<float>) == 36);
static_assert(sizeof(gwn_bvh_node<4, float>) == sizeof(gwnb_node4_f32));
static_assert(sizeof(gwn_bvh_child<float>) == sizeof(gwnb_child_f32));

template <int Width, int Order, gwn_real_type Real> struct gwn_bvh_moment_node;

template <int Width, gwn_real_type Real> struct gwn_bvh_moment_node<Width, 0, Real> {
    Real child_max_p_dist2[Width];
    Real child_average_x[Width];
    Real child_average_y[Width];
    Real child_average_z[Width];
    Real child_n_x[Width];
    Real child_n_y[Width];
    Real child_n_z[Width];
};

template <int Width, gwn_real_type Real> struct gwn_bvh_moment_node<Width, 1, Real> {
    Real child_max_p_dist2[Width];
    Real child_average_x[Width];
    Real child_average_y[Width];
    Real child_average_z[Width];
    Real child_n_x[Width];
    Real child_n_y[Width];
    Real child_n_z[Width];
    Real child_nij_xx[Width];
    Real child_nij_yy[Width];
    Real child_nij_zz[Width];
    Real child_nxy_nyx[Width];
    Real child_nyz_nzy[Width];
    Real child_nzx_nxz[Width];
};

template <int Width, gwn_real_type Real> struct gwn_bvh_moment_node<Width, 2, Real> {
    Real child_max_p_dist2[Width];
    Real child_average_x[Width];
    Real child_average_y[Width];
    Real child_average_z[Width];
    Real child_n_x[Width];
    Real child_n_y[Width];
    Real child_n_z[Width];
    Real child_nij_xx[Width];
    Real child_nij_yy[Width];
    Real child_nij_zz[Width];
    Real child_nxy_nyx[Width];
    Real child_nyz_nzy[Width];
    Real child_nzx_nxz[Width];
    Real child_nijk_xxx[Width];
    Real child_nijk_yyy[Width];
    Real child_nijk_zzz[Width];
    Real child_sum_permute_nxyz[Width];
    Real child_2nxxy_nyxx[Width];
    Real child_2nxxz_nzxx[Width];
    Real child_2nyyz_nzyy[Width];
    Real child_2nyyx_nxyy[Width];
    Real child_2nzzx_nxzz[Width];
    Real child_2nzzy_nyzz[Width];
};

template <int Order, gwn_real_type Real> using gwn_bvh4_moment_node = gwn_bvh_moment_node<4, Order, Real>;

template <int Width, gwn_real_type Real, gwn_index_type Index = std::uint32_t> struct gwn_bvh_accessor {
    static_assert(Width >= 2, "BVH accessor width must be at least 2.");
    using real_type = Real;
    using index_type = Index;
    static constexpr int k_width = Width;

    cuda::std::span<gwn_bvh_node<Width, Real>> nodes{};
    cuda::std::span<Index> primitive_indices{};
    cuda::std::span<gwn_bvh_triangle<Real>> triangles{};
    gwn_bvh_child<Real> root{};
    std::uint32_t internal_stack_bound = 0;
    std::uint32_t packed_stack_bound = 0;
    std::uint64_t revision = 0;

    [[nodiscard]] constexpr bool has_internal_root() const noexcept { return root.is_internal(); }
    [[nodiscard]] constexpr bool has_leaf_root() const noexcept { return root.is_leaf(); }
    [[nodiscard]] constexpr bool is_valid() const noexcept {
        if (revision == 0 || !root.is_valid() || primitive_indices.empty() ||
            primitive_indices.size() != triangles.size())
            return false;
        if (!gwn_span_has_storage(nodes) || !gwn_span_has_storage(primitive_indices) ||
            !gwn_span_has_storage(triangles))
            return false;
        std::uint64_t const off = root.offset();
        if (root.is_internal())
            return off < nodes.size();
        std::uint64_t const cnt = root.primitive_count();
        return off <= primitive_indices.size() && cnt <= primitive_indices.size() - off;
    }
};

template <gwn_real_type Real, gwn_index_type Index = std::uint32_t>
using gwn_bvh4_accessor = gwn_bvh_accessor<4, Real, Index>;

template <int Width, int Order, gwn_real_type Real, gwn_index_type Index = std::uint32_t>
struct gwn_bvh_moment_accessor {
    static_assert(Width >= 2, "BVH accessor width must be at least 2.");
    static_assert(Order == 0 || Order == 1 || Order == 2, "Taylor order must be 0, 1, or 2.");
    using real_type = Real;
    using index_type = Index;
    static constexpr int k_width = Width;
    static constexpr int k_order = Order;

    cuda::std::span<gwn_bvh_moment_node<Width, Order, Real>> nodes{};
    std::uint64_t bvh_revision = 0;

    [[nodiscard]] constexpr bool empty() const noexcept { return bvh_revision == 0; }
    [[nodiscard]] constexpr bool is_valid_for(gwn_bvh_accessor<Width, Real, Index> const &bvh) const noexcept {
        if (!bvh.is_valid() || bvh_revision != bvh.revision)
            return false;
        if (bvh.has_leaf_root())
            return nodes.empty();
        return gwn_span_has_storage(nodes) && nodes.size() == bvh.nodes.size();
    }
};

template <int Order, gwn_real_type Real, gwn_index_type Index = std::uint32_t>
using gwn_bvh4_moment_accessor = gwn_bvh_moment_accessor<4, Order, Real, Index>;

template <int Width, gwn_real_type Real = float, gwn_index_type Index = std::uint32_t> class gwn_bvh_object;
template <int Width, int Order, gwn_real_type Real = float, gwn_index_type Index = std::uint32_t>
class gwn_bvh_moment_object;

namespace detail {

template <int Width, gwn_real_type Real, gwn_index_type Index>
[[nodiscard]] inline gwnb_bvh4_f32 to_gwnb(gwn_bvh_accessor<Width, Real, Index> const &a, gwnb_bvh_aux *aux,
                                           std::uint64_t capacity) noexcept {
    gwnb_bvh4_f32 v{};
    if constexpr (Width == 4 && k_supported<Real, Index>) {
        v.nodes = reinterpret_cast<gwnb_node4_f32 *>(a.nodes.data());
        v.node_count = a.nodes.size();
        v.node_capacity = capacity > a.nodes.size() ? capacity : a.nodes.size();
        v.primitive_indices = a.primitive_indices.data();
        v.triangles = reinterpret_cast<gwnb_triangle_f32 *>(a.triangles.data());
        v.primitive_count = a.primitive_indices.size();
        static_assert(sizeof(v.root) == sizeof(a.root));
        __builtin_memcpy(static_cast<void *>(&v.root), static_cast<void const *>(&a.root), sizeof(v.root));
        v.internal_stack_bound = a.internal_stack_bound;
        v.packed_stack_bound = a.packed_stack_bound;
        v.revision = a.revision;
        v.aux = aux;
    }
    return v;
}

template <int Width, gwn_real_type Real, gwn_index_type Index>
inline void from_gwnb(gwnb_bvh4_f32 const &v, gwn_bvh_accessor<Width, Real, Index> &a) noexcept {
    if constexpr (Width == 4 && k_supported<Real, Index>) {
        a.nodes = cuda::std::span<gwn_bvh_node<Width, Real>>(reinterpret_cast<gwn_bvh_node<Width, Real> *>(v.nodes),
                                                             v.node_count);
        a.primitive_indices = cuda::std::span<Index>(v.primitive_indices, v.primitive_count);
        a.triangles = cuda::std::span<gwn_bvh_triangle<Real>>(
            reinterpret_cast<gwn_bvh_triangle<Real> *>(v.triangles), v.primitive_count);
        __builtin_memcpy(static_cast<void *>(&a.root), &v.root, sizeof(a.root));
        a.internal_stack_bound = v.internal_stack_bound;
        a.packed_stack_bound = v.packed_stack_bound;
        a.revision = v.revision;
    }
}

/// Access to the library handle inside owning objects (used by the free functions).
struct object_access {
    template <class Object> static gwnb_bvh_aux *&aux(Object &o) noexcept { return o.aux_; }
    template <class Object> static std::uint64_t &capacity(Object &o) noexcept { return o.capacity_; }
    template <class Object> static gwnb_moment_aux *&moment_aux(Object &o) noexcept { return o.aux_; }
};

} // namespace detail

/// Owning BVH: nodes, primitive order and triangle records in device memory.
template <int Width, gwn_real_type Real, gwn_index_type Index>
class gwn_bvh_object final : public gwn_noncopyable, public gwn_stream_mixin {
public:
    static_assert(Width >= 2, "BVH object width must be at least 2.");
    using real_type = Real;
    using index_type = Index;
    using accessor_type = gwn_bvh_accessor<Width, Real, Index>;

    gwn_bvh_object() = default;
    gwn_bvh_object(gwn_bvh_object &&other) noexcept { swap(*this, other); }
    gwn_bvh_object &operator=(gwn_bvh_object other) noexcept {
        swap(*this, other);
        return *this;
    }
    ~gwn_bvh_object() { clear(); }

    void clear() noexcept {
        if (accessor_.primitive_indices.data() != nullptr || aux_ != nullptr) {
            gwnb_bvh4_f32 v = detail::to_gwnb(accessor_, aux_, capacity_);
            gwnb_bvh4_release_f32(&v, detail::gwnb_stream(stream()));
        }
        accessor_ = accessor_type{};
        aux_ = nullptr;
        capacity_ = 0;
    }

    [[nodiscard]] accessor_type &accessor() noexcept { return accessor_; }
    [[nodiscard]] accessor_type const &accessor() const noexcept { return accessor_; }
    [[nodiscard]] bool has_data() const noexcept { return accessor_.is_valid(); }

    friend void swap(gwn_bvh_object &lhs, gwn_bvh_object &rhs) noexcept {
        using std::swap;
        swap(lhs.accessor_, rhs.accessor_);
        swap(lhs.aux_, rhs.aux_);
        swap(lhs.capacity_, rhs.capacity_);
        swap(static_cast<gwn_stream_mixin &>(lhs), static_cast<gwn_stream_mixin &>(rhs));
    }

private:
    friend struct detail::object_access;
    accessor_type accessor_{};
    gwnb_bvh_aux *aux_ = nullptr;
    std::uint64_t capacity_ = 0;
};

template <gwn_real_type Real = float, gwn_index_type Index = std::uint32_t>
using gwn_bvh4_object = gwn_bvh_object<4, Real, Index>;

/// Owning Taylor moment payload aligned to one BVH revision.
template <int Width, int Order, gwn_real_type Real, gwn_index_type Index>
class gwn_bvh_moment_object final : public gwn_noncopyable, public gwn_stream_mixin {
public:
    static_assert(Width >= 2, "BVH object width must be at least 2.");
    static_assert(Order == 0 || Order == 1 || Order == 2, "Taylor order must be 0, 1, or 2.");
    using real_type = Real;
    using index_type = Index;
    using accessor_type = gwn_bvh_moment_accessor<Width, Order, Real, Index>;

    gwn_bvh_moment_object() = default;
    gwn_bvh_moment_object(gwn_bvh_moment_object &&other) noexcept { swap(*this, other); }
    gwn_bvh_moment_object &operator=(gwn_bvh_moment_object other) noexcept {
        swap(*this, other);
        return *this;
    }
    ~gwn_bvh_moment_object() { clear(); }

    void clear() noexcept {
        if (accessor_.nodes.data() != nullptr || aux_ != nullptr) {
            gwnb_moment4_f32 v = view();
            gwnb_moment4_release_f32(&v, detail::gwnb_stream(stream()));
        }
        accessor_ = accessor_type{};
        aux_ = nullptr;
    }

    [[nodiscard]] accessor_type &accessor() noexcept { return accessor_; }
    [[nodiscard]] accessor_type const &accessor() const noexcept { return accessor_; }
    [[nodiscard]] bool has_data() const noexcept { return !accessor_.empty(); }

    /// The C-ABI view of this object (library use).
    [[nodiscard]] gwnb_moment4_f32 view() const noexcept {
        gwnb_moment4_f32 v{};
        v.order = Order;
        v.nodes = accessor_.nodes.data();
        v.node_count = accessor_.nodes.size();
        v.bvh_revision = accessor_.bvh_revision;
        v.aux = aux_;
        return v;
    }

    friend void swap(gwn_bvh_moment_object &lhs, gwn_bvh_moment_object &rhs) noexcept {
        using std::swap;
        swap(lhs.accessor_, rhs.accessor_);
        swap(lhs.aux_, rhs.aux_);
        swap(static_cast<gwn_stream_mixin &>(lhs), static_cast<gwn_stream_mixin &>(rhs));
    }

private:
    friend struct detail::object_access;
    accessor_type accessor_{};
    gwnb_moment_aux *aux_ = nullptr;
};

template <int Order, gwn_real_type Real = float, gwn_index_type Index = std::uint32_t>
using gwn_bvh4_moment_object = gwn_bvh_moment_object<4, Order, Real, Index>;

} // namespace gwn
