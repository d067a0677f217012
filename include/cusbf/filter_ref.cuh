// filter_ref.cuh -- device view of a filter's shards (drop-in for the
// reference's include/cusbf/filter_ref.cuh:21-115 and the shard layout of
// include/cusbf/detail/filter_impl.cuh:19-48).  A shard is 32 bytes: four
// little-endian uint64_t words; shard i of a filter with n shards holds the
// bits of every k-mer whose minimizer hash h has (uint32_t)(h & (n - 1)) == i.
#pragma once

#include <cstdint>

#include <cusbf/config.cuh>

namespace cusbf {

template <typename Config>
struct alignas(32) filter_block {
    static constexpr uint64_t wordCount = Config::blockWordCount;
    static constexpr uint64_t wordBits = Config::wordBits;
    static constexpr uint64_t sliceWidth = 64 / Config::hashCount;
    static constexpr bool useBitSlicing = sliceWidth >= 6;
    uint64_t words[wordCount];

    // Bit of word HashIndex % 4 addressed by hash HashIndex of `baseHash`
    // (filter_impl.cuh:37-48).
    template <uint64_t HashIndex>
    [[nodiscard]] constexpr __host__ __device__ static uint64_t sectorizedBitAddress(
        uint64_t baseHash) {
        static_assert(HashIndex < Config::hashCount, "Hash index out of range");
        if constexpr (useBitSlicing) {
            return (baseHash >> (sliceWidth * HashIndex)) & 63u;
        } else {
            constexpr uint64_t salts[16] = {
                0x9E3779B97F4A7C15ULL, 0xC2B2AE3D27D4EB4FULL, 0x165667B19E3779F9ULL,
                0x85EBCA77C2B2AE63ULL, 0x27D4EB2F165667C5ULL, 0x94D049BB133111EFULL,
                0xBF58476D1CE4E5B9ULL, 0xD6E8FEB86659FD93ULL, 0xA0761D6478BD642FULL,
                0xE7037ED1A0B428DBULL, 0x8EBC6AF09C88C6E3ULL, 0x589965CC75374CC3ULL,
                0x1D8E4E27C47D124FULL, 0xEB449C93FBBEA6B5ULL, 0xDB4F0B9175AE2165ULL,
                0xBBE056FDADE14B91ULL};
            return (baseHash * salts[HashIndex]) >> 58;
        }
    }
};

template <typename Config>
class filter_ref {
   public:
    using block_type = filter_block<Config>;
    __host__ __device__ constexpr filter_ref() noexcept : blocks_{}, num_blocks_{} {}
    __host__ __device__ constexpr filter_ref(block_type* blocks, uint64_t num_blocks) noexcept
        : blocks_(blocks), num_blocks_(num_blocks) {}
    [[nodiscard]] __host__ __device__ block_type* blocks() const noexcept { return blocks_; }
    [[nodiscard]] __host__ __device__ uint64_t num_blocks() const noexcept { return num_blocks_; }
    [[nodiscard]] __host__ __device__ static uint64_t shard_index(uint64_t minimizer_hash,
                                                                  uint64_t num_blocks) noexcept {
        return minimizer_hash & (num_blocks - 1);
    }
    [[nodiscard]] __host__ __device__ uint64_t shard_index(uint64_t minimizer_hash) const noexcept {
        return shard_index(minimizer_hash, num_blocks_);
    }

   private:
    block_type* blocks_{};
    uint64_t num_blocks_{};
};

}  // namespace cusbf
