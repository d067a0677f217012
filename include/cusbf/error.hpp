// error.hpp -- Result<T> error returns (drop-in for the reference's
// include/cusbf/error.hpp:19-269 of tdortman/cuSBF).
//
// Same vocabulary as the reference: Error is a variant of CudaError, IoError,
// FastxParseError, InvalidArgumentError and ResourceError with an
// ErrorCategory; Result<T> derives from cuda::std::expected<T, Error>;
// Err/Ok/cuda_try and the CUSBF_TRY / CUSBF_UNWRAP / CUSBF_CUDA_TRY /
// CUSBF_CUDA_ABORT macros behave as there.  detail::status_error maps a
// status of the C ABI (include/sbf_b200.h) to an Error.
#pragma once

#include <cuda_runtime.h>

#include <cuda/std/expected>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <format>
#include <source_location>
#include <stdexcept>
#include <string>
#include <string_view>
#include <utility>
#include <variant>

#include <sbf_b200.h>

namespace cusbf {

struct SourceLocation {
    std::string file;
    uint32_t line{};
    uint32_t column{};

    [[nodiscard]] static SourceLocation from(std::source_location loc) {
        return SourceLocation{loc.file_name(), static_cast<uint32_t>(loc.line()),
                              static_cast<uint32_t>(loc.column())};
    }
    [[nodiscard]] static SourceLocation fastx(std::string_view file, uint32_t line,
                                              uint32_t column) {
        return SourceLocation{std::string(file), line, column};
    }
    [[nodiscard]] std::string to_string() const { return std::format("{}:{}:{}", file, line, column); }
};

struct CudaError {
    cudaError_t code{};
    SourceLocation location;
    std::string message;
};
struct IoError {
    std::string message;
};
struct FastxParseError {
    SourceLocation location;
    std::string message;
};
struct InvalidArgumentError {
    std::string message;
};
struct ResourceError {
    std::string message;
};

enum class ErrorCategory : uint8_t { cuda, io, fastx_parse, invalid_argument, resource };

struct Error {
    std::variant<CudaError, IoError, FastxParseError, InvalidArgumentError, ResourceError> kind;

    [[nodiscard]] ErrorCategory category() const noexcept {
        return static_cast<ErrorCategory>(kind.index());
    }
    [[nodiscard]] const std::string& message() const noexcept {
        return std::visit([](const auto& e) -> const std::string& { return e.message; }, kind);
    }
    [[nodiscard]] const CudaError* as_cuda() const noexcept { return std::get_if<CudaError>(&kind); }
    [[nodiscard]] const IoError* as_io() const noexcept { return std::get_if<IoError>(&kind); }
    [[nodiscard]] const FastxParseError* as_fastx_parse() const noexcept {
        return std::get_if<FastxParseError>(&kind);
    }
    [[nodiscard]] const InvalidArgumentError* as_invalid_argument() const noexcept {
        return std::get_if<InvalidArgumentError>(&kind);
    }
    [[nodiscard]] const ResourceError* as_resource() const noexcept {
        return std::get_if<ResourceError>(&kind);
    }

    [[nodiscard]] static Error cuda(cudaError_t code,
                                    std::source_location loc = std::source_location::current()) {
        SourceLocation site = SourceLocation::from(loc);
        std::string msg = std::format("{}: {}", site.to_string(), cudaGetErrorString(code));
        return Error{CudaError{code, std::move(site), std::move(msg)}};
    }
    [[nodiscard]] static Error io(std::string message) { return Error{IoError{std::move(message)}}; }
    [[nodiscard]] static Error fastx_parse(SourceLocation site, std::string_view detail) {
        std::string msg = std::format("{}: {}", site.to_string(), detail);
        return Error{FastxParseError{std::move(site), std::move(msg)}};
    }
    [[nodiscard]] static Error invalid_argument(std::string message) {
        return Error{InvalidArgumentError{std::move(message)}};
    }
    [[nodiscard]] static Error resource(std::string message) {
        return Error{ResourceError{std::move(message)}};
    }
};

template <typename T>
struct [[nodiscard]] Result : cuda::std::expected<T, Error> {
    using cuda::std::expected<T, Error>::expected;
    [[nodiscard]] static Result ok(T value) { return Result(std::move(value)); }
    [[nodiscard]] static Result err(Error error) {
        return Result(cuda::std::unexpect, std::move(error));
    }
};

template <>
struct [[nodiscard]] Result<void> : cuda::std::expected<void, Error> {
    using cuda::std::expected<void, Error>::expected;
    [[nodiscard]] static Result ok() { return {}; }
    [[nodiscard]] static Result err(Error error) {
        return Result(cuda::std::unexpect, std::move(error));
    }
};

inline void require_void(const Result<void>& result) {
    if (!result) {
        std::fputs(result.error().message().c_str(), stderr);
        std::fputc('\n', stderr);
        std::abort();
    }
}

inline void cuda_abort_on_error(cudaError_t error,
                                std::source_location loc = std::source_location::current()) {
    if (error == cudaSuccess) return;
    std::fputs(Error::cuda(error, loc).message().c_str(), stderr);
    std::fputc('\n', stderr);
    std::abort();
}

[[nodiscard]] inline cuda::std::unexpected<Error> Err(Error error) {
    return cuda::std::unexpected<Error>(std::move(error));
}

[[nodiscard]] inline Result<void> Ok() noexcept { return Result<void>::ok(); }

[[nodiscard]] inline Result<void> cuda_try(
    cudaError_t error, std::source_location loc = std::source_location::current()) {
    if (error == cudaSuccess) return Ok();
    return Err(Error::cuda(error, loc));
}

namespace detail {

template <typename T>
[[nodiscard]] T try_unwrap_success(Result<T>& r) {
    return std::move(*r);
}
inline void try_unwrap_success(Result<void>&) {}

[[nodiscard]] inline cuda::std::unexpected<Error> propagate_error(const Error& e) {
    return cuda::std::unexpected<Error>(Error{e});
}

// Error for a non-zero status of the C ABI, with the library's message.
[[nodiscard]] inline Error status_error(int status) {
    std::string msg = sbf_last_error_message();
    switch (status) {
        case SBF_ERR_CUDA:
            return Error{CudaError{static_cast<cudaError_t>(sbf_last_cuda_error()),
                                   SourceLocation{"libsbf_b200", 0, 0}, std::move(msg)}};
        case SBF_ERR_IO:
            return Error::io(std::move(msg));
        case SBF_ERR_FASTX_PARSE: {
            const char* file = nullptr;
            uint32_t line = 0, col = 0;
            sbf_last_error_location(&file, &line, &col);
            return Error{FastxParseError{SourceLocation{file ? file : "", line, col}, std::move(msg)}};
        }
        case SBF_ERR_RESOURCE:
            return Error::resource(std::move(msg));
        default:
            return Error::invalid_argument(std::move(msg));
    }
}

}  // namespace detail
}  // namespace cusbf

#define CUSBF_TRY(expr)                                                     \
    ({                                                                      \
        auto _cusbf_result = (expr);                                        \
        if (!_cusbf_result) {                                               \
            return ::cusbf::detail::propagate_error(_cusbf_result.error()); \
        }                                                                   \
        ::cusbf::detail::try_unwrap_success(_cusbf_result);                 \
    })

#define CUSBF_UNWRAP(expr)                                             \
    ({                                                                 \
        auto _cusbf_result = (expr);                                   \
        if (!_cusbf_result) {                                          \
            throw std::runtime_error(_cusbf_result.error().message()); \
        }                                                              \
        ::cusbf::detail::try_unwrap_success(_cusbf_result);            \
    })

#define CUSBF_CUDA_ABORT(expr) ::cusbf::cuda_abort_on_error((expr))

#define CUSBF_CUDA_TRY(expr) CUSBF_TRY(::cusbf::cuda_try((expr)))
