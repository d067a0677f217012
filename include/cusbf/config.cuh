// config.cuh -- compile-time filter configuration (drop-in for the reference's
// include/cusbf/config.cuh:28-118 of tdortman/cuSBF).
//
// Config<K, S, M, HashCount, CudaBlockSize, Alphabet> fixes the k-mer, s-mer
// and minimizer widths and the hash count exactly as in the reference; the
// derived constants and static checks are the same.  CudaBlockSize is kept
// for source compatibility; the B200 engine chooses its own launch geometry.
#pragma once

#include <cstdint>

#include <cusbf/Alphabet.cuh>

namespace cusbf {

template <typename Config>
class filter;

namespace detail {
constexpr uint64_t bit_width_u64(uint64_t x) {
    uint64_t w = 0;
    while (x) {
        ++w;
        x >>= 1;
    }
    return w;
}
constexpr bool single_bit_u64(uint64_t x) { return x && !(x & (x - 1)); }
}  // namespace detail

template <uint16_t K_, uint16_t S_, uint16_t M_, uint64_t HashCount_ = 4,
          uint64_t CudaBlockSize_ = 256, Alphabet Alphabet_ = DnaAlphabet>
struct Config {
    using Alphabet = Alphabet_;
    static constexpr uint16_t k = K_;
    static constexpr uint16_t m = M_;
    static constexpr uint16_t s = S_;
    static constexpr uint64_t hashCount = HashCount_;
    static constexpr uint64_t alphabetSize = Alphabet::symbolCount;
    static constexpr uint64_t symbolWidth = Alphabet::symbolWidth;
    static constexpr uint64_t symbolBits = detail::bit_width_u64(alphabetSize - 1);
    static constexpr uint64_t symbolMask = (uint64_t{1} << symbolBits) - 1;
    static constexpr uint64_t filterBlockBits = 256;
    static constexpr uint64_t cudaBlockSize = CudaBlockSize_;
    static constexpr uint64_t wordBits = 64;
    static constexpr uint64_t blockWordCount = filterBlockBits / wordBits;
    static constexpr uint64_t minimizerSpan = k - m + 1;
    static constexpr uint64_t findereSpan = k - s + 1;
    static constexpr uint64_t insertGroupSize = blockWordCount;
    static constexpr uint64_t queryGroupSize = 1;
    static constexpr uint64_t maxRunKmers = cudaBlockSize;

    static_assert(k > 0, "k must be positive");
    static_assert(symbolWidth > 0, "alphabet symbolWidth must be positive");
    static_assert(m > 0 && m <= k, "m must satisfy 0 < m <= k");
    static_assert(s > 0 && s <= k, "s must satisfy 0 < s <= k");
    static_assert(k * symbolBits <= 64, "k-mer must fit in one packed uint64_t");
    static_assert(m * symbolBits <= 64, "m-mer must fit in one packed uint64_t");
    static_assert(s * symbolBits <= 64, "s-mer must fit in one packed uint64_t");
    static_assert(hashCount > 0, "At least one Bloom hash is required");
    static_assert(hashCount <= 16, "This implementation provides 16 multiplicative salts");
    static_assert(hashCount >= blockWordCount, "Sectorized layout requires hashCount >= blockWordCount");
    static_assert(hashCount % blockWordCount == 0, "Hash count must distribute evenly across shard words");
    static_assert(cudaBlockSize % 32 == 0, "CUDA block size must be a multiple of one warp");
    static_assert(detail::single_bit_u64(filterBlockBits), "Filter block size must be a power of two");
};

}  // namespace cusbf
