#pragma once

/// \file gwn_eigen_bridge.cuh
/// \brief gwn_upload_geometry_from_eigen: N x 3 vertex and M x 3 triangle matrices to an uploaded
/// SoA geometry.
///
/// Same name, arguments, checks and messages as smallgwn's include/gwn/gwn_eigen_bridge.cuh:26-132,
/// without its Eigen and TBB requirements: the matrices are taken as any type with `rows()`,
/// `cols()` and `operator()(row, col)` (Eigen's MatrixBase, Map and Block qualify, as do row-major
/// and column-major storage and expressions), and the conversion runs on std::thread workers.
/// Index entries may be integer or floating point; a floating-point entry must be finite and
/// integer-valued. Every index must lie in [0, vertex_count).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <exception>
#include <limits>
#include <memory>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>

#include "gwn_geometry.cuh"

namespace gwn {

namespace detail {

/// Runs body(begin, end) over [0, count) on up to hardware_concurrency threads (one chunk per
/// thread; small ranges stay on the calling thread).
template <class Body> void host_parallel_for(std::size_t const count, Body &&body) {
    constexpr std::size_t k_serial = std::size_t(1) << 16;
    unsigned const hw = std::max(1u, std::thread::hardware_concurrency());
    std::size_t const workers = count < k_serial ? 1 : std::min<std::size_t>(hw, (count + k_serial - 1) / k_serial);
    if (workers <= 1) {
        body(std::size_t(0), count);
        return;
    }
    std::size_t const chunk = (count + workers - 1) / workers;
    std::vector<std::thread> threads;
    threads.reserve(workers - 1);
    try {
        for (std::size_t w = 1; w < workers; ++w) {
            std::size_t const b = w * chunk, e = std::min(count, b + chunk);
            if (b < e)
                threads.emplace_back([&body, b, e] { body(b, e); });
        }
    } catch (...) {
        for (auto &t : threads) // a thread that could not start: finish the started ones, then report
            t.join();
        throw;
    }
    body(std::size_t(0), std::min(count, chunk));
    for (auto &t : threads)
        t.join();
}

/// One matrix entry as an index in [0, vertex_count) (false when it is not one).
template <gwn_index_type Index, class Value>
[[nodiscard]] bool eigen_index(Value const value, std::size_t const vertex_count, Index &out) noexcept {
    using V = std::decay_t<Value>;
    std::uint64_t u = 0;
    if constexpr (std::is_floating_point_v<V>) {
        if (!std::isfinite(value) || std::floor(value) != value || value < V(0) ||
            value >= V(18446744073709551616.0))
            return false;
        u = static_cast<std::uint64_t>(value);
    } else {
        if constexpr (std::is_signed_v<V>) {
            if (value < V(0))
                return false;
        }
        u = static_cast<std::uint64_t>(value);
    }
    if (u >= vertex_count || u > static_cast<std::uint64_t>(std::numeric_limits<Index>::max()))
        return false;
    out = static_cast<Index>(u);
    return true;
}

} // namespace detail

/// Converts `vertices` (N x 3) and `triangles` (M x 3) to SoA arrays and uploads them with
/// gwn_upload_geometry; replaces \p object only on success.
template <gwn_real_type Real = float, gwn_index_type Index = std::uint32_t, class MatrixV, class MatrixF>
[[nodiscard]] gwn_status gwn_upload_geometry_from_eigen(gwn_geometry_object<Real, Index> &object,
                                                        MatrixV const &vertices, MatrixF const &triangles,
                                                        cudaStream_t const stream = gwn_default_stream()) noexcept try {
    if (vertices.cols() != 3 || triangles.cols() != 3)
        return gwn_status::invalid_argument("Eigen inputs must be Nx3 vertices and Mx3 triangles.");
    auto const vertex_rows = static_cast<std::int64_t>(vertices.rows());
    auto const triangle_rows = static_cast<std::int64_t>(triangles.rows());
    if (vertex_rows < 0 || triangle_rows < 0)
        return gwn_status::invalid_argument("Eigen inputs cannot have negative sizes.");
    auto const nv = static_cast<std::size_t>(vertex_rows);
    auto const nt = static_cast<std::size_t>(triangle_rows);
    if (nv > 0 && nv - 1 > static_cast<std::size_t>(std::numeric_limits<Index>::max()))
        return gwn_status::invalid_argument("Vertex count exceeds index range.");

    std::vector<Real> x(nv), y(nv), z(nv);
    detail::host_parallel_for(nv, [&](std::size_t const b, std::size_t const e) {
        for (std::size_t i = b; i < e; ++i) {
            auto const r = static_cast<std::int64_t>(i);
            x[i] = static_cast<Real>(vertices(r, 0));
            y[i] = static_cast<Real>(vertices(r, 1));
            z[i] = static_cast<Real>(vertices(r, 2));
        }
    });

    std::vector<Index> i0(nt), i1(nt), i2(nt);
    std::atomic<bool> bad{false};
    detail::host_parallel_for(nt, [&](std::size_t const b, std::size_t const e) {
        for (std::size_t i = b; i < e; ++i) {
            auto const r = static_cast<std::int64_t>(i);
            if (!(detail::eigen_index<Index>(triangles(r, 0), nv, i0[i]) &&
                  detail::eigen_index<Index>(triangles(r, 1), nv, i1[i]) &&
                  detail::eigen_index<Index>(triangles(r, 2), nv, i2[i])))
                bad.store(true, std::memory_order_relaxed);
        }
    });
    if (bad.load(std::memory_order_relaxed))
        return gwn_status::invalid_argument("Eigen triangle indices must be integer-valued in [0, vertex_count).");

    return gwn_upload_geometry(object, gwn_host_span<Real const>(x.data(), nv), gwn_host_span<Real const>(y.data(), nv),
                               gwn_host_span<Real const>(z.data(), nv), gwn_host_span<Index const>(i0.data(), nt),
                               gwn_host_span<Index const>(i1.data(), nt), gwn_host_span<Index const>(i2.data(), nt),
                               stream);
} catch (std::exception const &) {
    return gwn_status::internal_error("Unhandled std::exception in gwn_upload_geometry_from_eigen.");
} catch (...) {
    return gwn_status::internal_error("Unhandled unknown exception in gwn_upload_geometry_from_eigen.");
}

} // namespace gwn
