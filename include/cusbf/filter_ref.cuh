// filter_ref.cuh -- device view of a filter's shards for callers' own kernels
// (drop-in for the reference's include/cusbf/filter_ref.cuh:21-115 and the
// shard layout of
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

    // The same bit address for a run-time hash index j < hashCount.
    [[nodiscard]] constexpr __host__ __device__ static uint64_t sectorizedBitAddress(
        uint64_t baseHash, uint64_t j) {
        if constexpr (useBitSlicing) {
            return (baseHash >> (sliceWidth * j)) & 63u;
        } else {
            constexpr uint64_t salts[16] = {
                0x9E3779B97F4A7C15ULL, 0xC2B2AE3D27D4EB4FULL, 0x165667B19E3779F9ULL,
                0x85EBCA77C2B2AE63ULL, 0x27D4EB2F165667C5ULL, 0x94D049BB133111EFULL,
                0xBF58476D1CE4E5B9ULL, 0xD6E8FEB86659FD93ULL, 0xA0761D6478BD642FULL,
                0xE7037ED1A0B428DBULL, 0x8EBC6AF09C88C6E3ULL, 0x589965CC75374CC3ULL,
                0x1D8E4E27C47D124FULL, 0xEB449C93FBBEA6B5ULL, 0xDB4F0B9175AE2165ULL,
                0xBBE056FDADE14B91ULL};
            return (baseHash * salts[j]) >> 58;
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

    // Findere membership of one window against its shard's four words
    // (filter_ref.cuh:70-87): true when every one of the k-s+1 s-mers of the
    // packed k-mer (Config::symbolBits per symbol, earliest symbol in the
    // highest bits) has all of its hashCount bits set.  The s-mer hash is
    // x * 0x9e3779b97f4a7c15 followed by h ^= h >> 33 (hashutil.cuh:192-196).
    [[nodiscard]] __device__ static bool sectorized_contains_packed_kmer(
        uint64_t packed_kmer, const uint64_t* shard_words) {
        constexpr uint64_t kSmerBits = uint64_t{Config::s} * Config::symbolBits;
        constexpr uint64_t kSmerMask =
            kSmerBits >= 64 ? ~uint64_t{0} : (uint64_t{1} << kSmerBits) - 1;
        bool present = true;
#pragma unroll
        for (uint64_t o = 0; o < Config::findereSpan; ++o) {
            const uint64_t shift = Config::symbolBits * (Config::k - o - Config::s);
            uint64_t h = ((packed_kmer >> shift) & kSmerMask) * 0x9e3779b97f4a7c15ULL;
            h ^= h >> 33;
#pragma unroll
            for (uint64_t j = 0; j < Config::hashCount; ++j) {
                const uint64_t bit = block_type::sectorizedBitAddress(h, j);
                present &= ((shard_words[j % Config::blockWordCount] >> bit) & 1u) != 0;
            }
        }
        return present;
    }

    // ORs the non-zero word masks of one super-k-mer run into `block` with one
    // 64-bit atomic per word (filter_ref.cuh:94-108).
    __device__ void apply_word_masks(block_type& block, uint64_t m0, uint64_t m1, uint64_t m2,
                                     uint64_t m3) const {
        auto* w = reinterpret_cast<unsigned long long*>(block.words);
        if (m0) atomicOr(w + 0, static_cast<unsigned long long>(m0));
        if (m1) atomicOr(w + 1, static_cast<unsigned long long>(m1));
        if (m2) atomicOr(w + 2, static_cast<unsigned long long>(m2));
        if (m3) atomicOr(w + 3, static_cast<unsigned long long>(m3));
    }

   private:
    block_type* blocks_{};
    uint64_t num_blocks_{};
};

}  // namespace cusbf
