// dense_packed.hpp -- 2-bit dense packing (drop-in for the reference's
// include/cusbf/dense_packed.hpp:20-74): 32 symbols per uint64_t word,
// symbol t at bits [2(t%32), 2(t%32)+2) of word t/32, invalid bytes stored as
// their low two code bits.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string_view>
#include <vector>

#include <cusbf/config.cuh>
#include <cusbf/error.hpp>

namespace cusbf {

template <typename Config>
[[nodiscard]] constexpr uint64_t dense_packed_word_count(uint64_t num_symbols) {
    constexpr uint64_t per = 64 / Config::symbolBits;
    return (num_symbols + per - 1) / per;
}

template <typename Config>
[[nodiscard]] constexpr uint64_t dense_packed_kmer_count(uint64_t num_symbols) {
    return num_symbols < Config::k ? 0 : num_symbols - Config::k + 1;
}

template <typename Config>
[[nodiscard]] std::vector<uint64_t> pack_dense_sequence(std::string_view sequence) {
    static_assert(Config::symbolBits == 2 && Config::symbolWidth == 1,
                  "the B200 engine packs the 2-bit DNA alphabet");
    std::vector<uint64_t> words(dense_packed_word_count<Config>(sequence.size()), 0);
    if (!sequence.empty()) sbf_pack_dense_host(sequence.data(), sequence.size(), words.data());
    return words;
}

template <typename Config>
inline void pack_dense_sequence_device(const char* d_sequence, uint64_t num_symbols,
                                       uint64_t* d_words, cudaStream_t stream = {}) {
    if (num_symbols == 0) return;
    const int s = sbf_pack_dense_device(d_sequence, num_symbols, d_words,
                                        reinterpret_cast<sbf_stream_t>(stream));
    if (s != SBF_OK) throw std::runtime_error(detail::status_error(s).message());
}

}  // namespace cusbf
