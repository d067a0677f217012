// dense_packed.hpp -- dense packing (drop-in for the reference's
// include/cusbf/dense_packed.hpp:20-74): 64 / symbolBits symbols per uint64_t
// word (32 for DNA), symbol t at bits [b(t%per), b(t%per)+b) of word t/per,
// invalid symbols stored as their low symbolBits bits.
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
    const uint64_t num_symbols = sequence.size() / Config::symbolWidth;
    std::vector<uint64_t> words(dense_packed_word_count<Config>(num_symbols), 0);
    if (num_symbols == 0) return words;
    const int s = sbf_pack_dense_host_for(detail::alphabet_id<typename Config::Alphabet>(),
                                          sequence.data(), num_symbols, words.data());
    if (s != SBF_OK) throw std::runtime_error(detail::status_error(s).message());
    return words;
}

template <typename Config>
inline void pack_dense_sequence_device(const char* d_sequence, uint64_t num_symbols,
                                       uint64_t* d_words, cudaStream_t stream = {}) {
    if (num_symbols == 0) return;
    const int s = sbf_pack_dense_device_for(detail::alphabet_id<typename Config::Alphabet>(),
                                            d_sequence, num_symbols, d_words,
                                            reinterpret_cast<sbf_stream_t>(stream));
    if (s != SBF_OK) throw std::runtime_error(detail::status_error(s).message());
}

}  // namespace cusbf
