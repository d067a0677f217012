// Alphabet.cuh -- byte-to-symbol alphabets (drop-in for the reference's
// include/cusbf/Alphabet.cuh:95-220).  The concept and the three alphabets
// keep the reference's names, constants and encodings so configurations
// written against the reference compile unchanged; the B200 engine executes
// the DNA alphabet (A0 C1 T2 G3, case-insensitive, invalid 0xFF).
#pragma once

#include <concepts>
#include <cstdint>

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif
#endif

namespace cusbf {

template <typename T>
concept Alphabet = requires(const char* input) {
    { T::symbolCount } -> std::convertible_to<uint64_t>;
    { T::symbolWidth } -> std::convertible_to<uint64_t>;
    { T::invalidSymbol } -> std::convertible_to<uint8_t>;
    { T::separator } -> std::convertible_to<uint8_t>;
    { T::validBytes } -> std::convertible_to<const char*>;
    { T::encode(input) } -> std::same_as<uint8_t>;
} && requires {
    requires T::symbolCount > 0 && T::symbolCount <= 255;
    requires T::symbolWidth > 0;
};

struct DnaAlphabet {
    static constexpr uint64_t symbolWidth = 1;
    static constexpr uint64_t symbolCount = 4;
    static constexpr uint8_t invalidSymbol = 0xFFu;
    static constexpr uint8_t separator = 'N';
    static constexpr char validBytes[] = "ACGT";

    [[nodiscard]] constexpr __host__ __device__ __forceinline__ static uint8_t encode(
        const char* input) {
        const auto byte = static_cast<uint8_t>(input[0]);
        const uint8_t upper = byte & 0xDFu;
        const bool valid = upper == 'A' || upper == 'C' || upper == 'G' || upper == 'T';
        return valid ? static_cast<uint8_t>((byte >> 1u) & 3u) : invalidSymbol;
    }
};

struct DnaTripletAlphabet {
    static constexpr uint64_t symbolWidth = 3;
    static constexpr uint64_t symbolCount = 64;
    static constexpr uint8_t invalidSymbol = 0xFFu;
    static constexpr uint8_t separator = 'N';
    static constexpr char validBytes[] = "ACGT";

    [[nodiscard]] constexpr __host__ __device__ __forceinline__ static uint8_t encode(
        const char* input) {
        const uint8_t a = DnaAlphabet::encode(input + 0);
        const uint8_t b = DnaAlphabet::encode(input + 1);
        const uint8_t c = DnaAlphabet::encode(input + 2);
        if (a == invalidSymbol || b == invalidSymbol || c == invalidSymbol) return invalidSymbol;
        return static_cast<uint8_t>((a << 4u) | (b << 2u) | c);
    }
};

struct ProteinAlphabet {
    static constexpr uint64_t symbolWidth = 1;
    static constexpr uint64_t symbolCount = 26;
    static constexpr uint8_t invalidSymbol = 0xFFu;
    static constexpr uint8_t separator = '*';
    static constexpr char validBytes[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZ";

    [[nodiscard]] constexpr __host__ __device__ __forceinline__ static uint8_t encode(
        const char* input) {
        const uint8_t letter = static_cast<uint8_t>((static_cast<uint8_t>(input[0]) & 0xDFu) - 'A');
        return letter < 26 ? letter : invalidSymbol;
    }
};

namespace detail {
// Alphabet id understood by the C ABI (SBF_ALPHABET_*), or -1.
template <typename A>
constexpr int alphabet_id() {
    if constexpr (std::same_as<A, DnaAlphabet>) return 0;
    if constexpr (std::same_as<A, DnaTripletAlphabet>) return 1;
    if constexpr (std::same_as<A, ProteinAlphabet>) return 2;
    return -1;
}
}  // namespace detail

}  // namespace cusbf
