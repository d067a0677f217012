// device_span.cuh -- span over device memory (drop-in for the reference's
// include/cusbf/device_span.cuh:21-33).
#pragma once

#include <cuda/std/span>

#include <type_traits>

namespace cusbf {

template <typename T>
struct device_span : cuda::std::span<T> {
    using cuda::std::span<T>::span;

    template <typename U>
        requires std::is_convertible_v<U (*)[], T (*)[]>
    constexpr explicit device_span(device_span<U> other) noexcept
        : cuda::std::span<T>(other.data(), other.size()) {}
};

}  // namespace cusbf
