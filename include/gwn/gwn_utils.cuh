#pragma once

/// \file gwn_utils.cuh
/// \brief Status, spans and stream binding of the drop-in API (host code; no device code needed).
///
/// Same names and semantics as smallgwn's include/gwn/gwn_utils.cuh:20-396 (gwn_status,
/// gwn_error, gwn_host_span / gwn_device_span, gwn_stream_mixin, GWN_RETURN_ON_ERROR). The
/// implementation behind every operation is libgwnb.so (include/gwnb.h).

#include <cuda/std/span>
#include <cuda_runtime_api.h>

#include <concepts>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <source_location>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>

#include "../gwnb.h"

namespace gwn {

template <class Real>
concept gwn_real_type = std::floating_point<Real>;

template <class Index>
concept gwn_index_type = std::same_as<Index, std::uint32_t> || std::same_as<Index, std::uint64_t>;

class gwn_noncopyable {
protected:
    constexpr gwn_noncopyable() noexcept = default;
    ~gwn_noncopyable() = default;
    gwn_noncopyable(gwn_noncopyable &&) noexcept = default;
    gwn_noncopyable &operator=(gwn_noncopyable &&) noexcept = default;

public:
    gwn_noncopyable(gwn_noncopyable const &) = delete;
    gwn_noncopyable &operator=(gwn_noncopyable const &) = delete;
};

[[nodiscard]] inline cudaStream_t gwn_default_stream() noexcept { return cudaStreamLegacy; }

class gwn_stream_mixin {
public:
    gwn_stream_mixin() noexcept = default;
    explicit gwn_stream_mixin(cudaStream_t const stream) noexcept : stream_{stream} {}
    [[nodiscard]] cudaStream_t stream() const noexcept { return stream_; }
    void set_stream(cudaStream_t const stream) noexcept { stream_ = stream; }
    friend void swap(gwn_stream_mixin &lhs, gwn_stream_mixin &rhs) noexcept {
        using std::swap;
        swap(lhs.stream_, rhs.stream_);
    }

private:
    cudaStream_t stream_{gwn_default_stream()};
};

/// Non-owning host-memory view.
template <class T> class gwn_host_span final {
public:
    constexpr gwn_host_span() noexcept = default;
    constexpr gwn_host_span(T *const data, std::size_t const size) noexcept : span_(data, size) {}
    explicit constexpr gwn_host_span(cuda::std::span<T> const span) noexcept : span_(span) {}
    template <class U>
        requires std::is_convertible_v<U (*)[], T (*)[]>
    constexpr gwn_host_span(gwn_host_span<U> const other) noexcept : span_(other.data(), other.size()) {}
    [[nodiscard]] constexpr T *data() const noexcept { return span_.data(); }
    [[nodiscard]] constexpr std::size_t size() const noexcept { return span_.size(); }
    [[nodiscard]] constexpr bool empty() const noexcept { return span_.empty(); }

private:
    cuda::std::span<T> span_{};
};

/// Non-owning device-accessible view.
template <class T> class gwn_device_span final {
public:
    constexpr gwn_device_span() noexcept = default;
    constexpr gwn_device_span(T *const data, std::size_t const size) noexcept : span_(data, size) {}
    explicit constexpr gwn_device_span(cuda::std::span<T> const span) noexcept : span_(span) {}
    template <class U>
        requires std::is_convertible_v<U (*)[], T (*)[]>
    constexpr gwn_device_span(gwn_device_span<U> const other) noexcept : span_(other.data(), other.size()) {}
    [[nodiscard]] constexpr T *data() const noexcept { return span_.data(); }
    [[nodiscard]] constexpr std::size_t size() const noexcept { return span_.size(); }
    [[nodiscard]] constexpr bool empty() const noexcept { return span_.empty(); }

private:
    cuda::std::span<T> span_{};
};

template <class T>
[[nodiscard]] constexpr bool gwn_span_has_storage(cuda::std::span<T> const span) noexcept {
    return span.empty() || span.data() != nullptr;
}

template <gwn_index_type Index> [[nodiscard]] constexpr Index gwn_invalid_index() noexcept {
    return std::numeric_limits<Index>::max();
}
template <gwn_index_type Index> [[nodiscard]] constexpr bool gwn_is_invalid_index(Index const i) noexcept {
    return i == gwn_invalid_index<Index>();
}
template <gwn_index_type Index> [[nodiscard]] constexpr bool gwn_is_valid_index(Index const i) noexcept {
    return !gwn_is_invalid_index(i);
}
template <gwn_index_type Index>
[[nodiscard]] constexpr bool gwn_index_in_bounds(Index const i, std::size_t const bound) noexcept {
    return gwn_is_valid_index(i) && static_cast<std::size_t>(i) < bound;
}

enum class gwn_error {
    success = 0,
    invalid_argument,
    cuda_runtime_error,
    internal_error,
};

/// Status returned by every public host function.
class gwn_status {
public:
    gwn_status() noexcept = default;
    [[nodiscard]] static gwn_status ok() noexcept { return gwn_status(); }
    [[nodiscard]] static gwn_status invalid_argument(std::string message) noexcept {
        return gwn_status(gwn_error::invalid_argument, std::move(message));
    }
    [[nodiscard]] static gwn_status internal_error(std::string message = "Internal error.") noexcept {
        return gwn_status(gwn_error::internal_error, std::move(message));
    }
    [[nodiscard]] static gwn_status cuda_runtime_error(
        cudaError_t const result, std::source_location const location = std::source_location::current(),
        std::string message = "CUDA API call failed."
    ) noexcept {
        char const *const name = cudaGetErrorName(result);
        char const *const text = cudaGetErrorString(result);
        message += std::string{" [cuda_error="} + std::to_string(static_cast<int>(result)) + " (" +
                   (name != nullptr ? name : "unknown") + "): \"" + (text != nullptr ? text : "unknown") + "\"]";
        return gwn_status(gwn_error::cuda_runtime_error, std::move(message), location);
    }
    [[nodiscard]] bool is_ok() const noexcept { return error_ == gwn_error::success; }
    [[nodiscard]] gwn_error error() const noexcept { return error_; }
    [[nodiscard]] std::source_location location() const noexcept { return location_; }
    [[nodiscard]] bool has_location() const noexcept { return location_.line() != 0; }
    [[nodiscard]] std::string const &message() const noexcept { return message_; }

private:
    gwn_status(gwn_error const e, std::string m) noexcept : error_{e}, message_{std::move(m)} {}
    gwn_status(gwn_error const e, std::string m, std::source_location const l) noexcept
        : error_{e}, location_{l}, message_{std::move(m)} {}

    gwn_error error_{gwn_error::success};
    std::source_location location_{};
    std::string message_{};
};

#ifndef GWN_RETURN_ON_ERROR
#define GWN_RETURN_ON_ERROR(expr)                                                                  \
    do {                                                                                           \
        ::gwn::gwn_status const gwn_status_result_ = (expr);                                       \
        if (!gwn_status_result_.is_ok())                                                           \
            return gwn_status_result_;                                                             \
    } while (false)
#endif

inline void gwn_throw_if_error(gwn_status const &status) {
    if (status.is_ok())
        return;
    std::string message = status.message();
    if (status.has_location())
        message += std::string{" at "} + status.location().file_name() + ":" + std::to_string(status.location().line());
    throw std::runtime_error(message);
}

[[nodiscard]] inline gwn_status
gwn_cuda_to_status(cudaError_t const result, std::source_location const location = std::source_location::current()) noexcept {
    if (result == cudaSuccess)
        return gwn_status::ok();
    return gwn_status::cuda_runtime_error(result, location);
}

namespace detail {

/// Translate a libgwnb status code into gwn_status.
[[nodiscard]] inline gwn_status gwnb_to_status(int const rc) noexcept {
    switch (rc) {
    case GWNB_OK: return gwn_status::ok();
    case GWNB_INVALID_ARGUMENT: return gwn_status::invalid_argument(gwnb_last_error_message());
    case GWNB_CUDA_RUNTIME_ERROR:
        return gwn_status::cuda_runtime_error(static_cast<cudaError_t>(gwnb_last_cuda_error()),
                                              std::source_location::current(), gwnb_last_error_message());
    default: return gwn_status::internal_error(gwnb_last_error_message());
    }
}

[[nodiscard]] inline gwnb_stream_t gwnb_stream(cudaStream_t const s) noexcept {
    return reinterpret_cast<gwnb_stream_t>(s);
}

template <class Real, class Index> inline constexpr bool k_supported = std::is_same_v<Real, float> &&
                                                                       std::is_same_v<Index, std::uint32_t>;

[[nodiscard]] inline gwn_status unsupported_instantiation() noexcept {
    return gwn_status::invalid_argument(
        "unsupported instantiation: this library provides Width = 4, Real = float, Index = uint32_t.");
}

} // namespace detail

/// Device memory the library's pool holds from the driver and the part of it in live allocations
/// (current device). No smallgwn counterpart: its allocations use the CUDA defaults.
[[nodiscard]] inline gwn_status gwn_memory_stats(std::uint64_t &reserved_bytes, std::uint64_t &used_bytes) noexcept {
    return detail::gwnb_to_status(gwnb_memory_stats(&reserved_bytes, &used_bytes));
}

/// Returns the pool's cached device memory to the driver down to keep_bytes (or what is in use).
[[nodiscard]] inline gwn_status gwn_memory_trim(std::uint64_t const keep_bytes = 0) noexcept {
    return detail::gwnb_to_status(gwnb_memory_trim(keep_bytes));
}

/// Kernel launches the library has issued in this process (a launch recorded into a CUDA graph
/// counts once, when captured).
[[nodiscard]] inline std::uint64_t gwn_launch_count() noexcept { return gwnb_launch_count(); }

} // namespace gwn
