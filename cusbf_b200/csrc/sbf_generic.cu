// sbf_generic.cu -- the runtime-parameterised kernels (sbf_generic.cuh)
// compiled into the library for every configuration without specialised
// kernels, and dense packing for every alphabet.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/sbf_b200.h"
#include "sbf_device.cuh"
#include "sbf_generic.cuh"
#include "sbf_host.h"
#include "sbf_internal.h"

namespace sbf {

static_assert(kAlphabetDna == SBF_ALPHABET_DNA && kAlphabetTriplet == SBF_ALPHABET_DNA_TRIPLET &&
                  kAlphabetProtein == SBF_ALPHABET_PROTEIN,
              "alphabet ids match the C ABI");

namespace {

template <bool Q, bool D, bool R>
const void* generic_ptr() {
    return reinterpret_cast<const void*>(&generic_kernel<RuntimeGen, Q, D, R>);
}

const KernelSet kGeneric = {
    0, 0, 0, 0,
    generic_ptr<false, false, false>(),
    generic_ptr<true, false, false>(),
    generic_ptr<false, true, false>(),
    generic_ptr<true, true, false>(),
    generic_ptr<false, false, true>(),
    generic_ptr<true, false, true>(),
    0,
    0,
};

// Dense packing for any alphabet (pack_dense_sequence_kernel,
// detail/dense_packed.cuh:62-90): one thread per word, 64 / bits symbols per
// word, invalid symbols stored as their low `bits` bits.
__global__ void pack_dense_generic_kernel(GenericCfg c, const uint8_t* seq, uint64_t num_symbols,
                                          uint64_t* words) {
    const uint32_t per_word = 64u / c.bits;
    const uint64_t n_words = (num_symbols + per_word - 1) / per_word;
    const uint64_t mask = (uint64_t{1} << c.bits) - 1;
    for (uint64_t w = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; w < n_words;
         w += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t out = 0;
        const uint64_t first = w * per_word;
        for (uint32_t t = 0; t < per_word && first + t < num_symbols; ++t)
            out |= (encode_symbol(c, seq + (first + t) * c.width) & mask) << (t * c.bits);
        words[w] = out;
    }
}

}  // namespace

const KernelSet* generic_kernels() { return &kGeneric; }

bool alphabet_geometry(int alphabet, uint32_t* bits, uint32_t* width) {
    switch (alphabet) {
        case SBF_ALPHABET_DNA: *bits = 2; *width = 1; return true;
        case SBF_ALPHABET_PROTEIN: *bits = 5; *width = 1; return true;
        case SBF_ALPHABET_DNA_TRIPLET: *bits = 6; *width = 3; return true;
        default: return false;
    }
}

}  // namespace sbf

using sbf::GenericCfg;

extern "C" uint64_t sbf_dense_packed_word_count_for(int alphabet, uint64_t num_symbols) {
    uint32_t bits = 0, width = 0;
    if (!sbf::alphabet_geometry(alphabet, &bits, &width)) return 0;
    const uint64_t per = 64u / bits;
    return (num_symbols + per - 1) / per;
}

extern "C" int sbf_pack_dense_host_for(int alphabet, const char* h_seq, uint64_t num_symbols,
                                       uint64_t* h_words) {
    uint32_t bits = 0, width = 0;
    if (!sbf::alphabet_geometry(alphabet, &bits, &width))
        return sbf::set_error(SBF_ERR_INVALID_ARGUMENT, "unknown alphabet %d", alphabet);
    if (num_symbols == 0) return SBF_OK;
    if (!h_seq || !h_words) return sbf::set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    const uint64_t per = 64u / bits, mask = (uint64_t{1} << bits) - 1;
    const uint64_t n_words = (num_symbols + per - 1) / per;
    for (uint64_t w = 0; w < n_words; ++w) h_words[w] = 0;
    auto dna = [](uint8_t b) -> uint8_t {
        const uint8_t u = b & 0xDFu;
        return (u == 'A' || u == 'C' || u == 'G' || u == 'T') ? ((b >> 1) & 3u) : 0xFFu;
    };
    for (uint64_t t = 0; t < num_symbols; ++t) {
        const auto* p = reinterpret_cast<const uint8_t*>(h_seq) + t * width;
        uint8_t e;
        if (alphabet == SBF_ALPHABET_PROTEIN) {
            const uint8_t idx = static_cast<uint8_t>((p[0] & 0xDFu) - 'A');
            e = idx < 26 ? idx : 0xFFu;
        } else if (alphabet == SBF_ALPHABET_DNA_TRIPLET) {
            const uint8_t a = dna(p[0]), b = dna(p[1]), c = dna(p[2]);
            e = (a == 0xFF || b == 0xFF || c == 0xFF) ? 0xFFu
                                                       : static_cast<uint8_t>((a << 4) | (b << 2) | c);
        } else {
            e = dna(p[0]);
        }
        h_words[t / per] |= (e & mask) << ((t % per) * bits);
    }
    return SBF_OK;
}

extern "C" int sbf_pack_dense_device_for(int alphabet, const char* d_seq, uint64_t num_symbols,
                                         uint64_t* d_words, sbf_stream_t stream) {
    uint32_t bits = 0, width = 0;
    if (!sbf::alphabet_geometry(alphabet, &bits, &width))
        return sbf::set_error(SBF_ERR_INVALID_ARGUMENT, "unknown alphabet %d", alphabet);
    if (num_symbols == 0) return SBF_OK;
    if (!d_seq || !d_words) return sbf::set_error(SBF_ERR_INVALID_ARGUMENT, "null device pointer");
    const uint64_t n_words = sbf_dense_packed_word_count_for(alphabet, num_symbols);
    const GenericCfg c{0, 0, 0, 0, bits, width, static_cast<uint32_t>(alphabet)};
    const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((n_words + 255) / 256, 65535));
    sbf::pack_dense_generic_kernel<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        c, reinterpret_cast<const uint8_t*>(d_seq), num_symbols, d_words);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return sbf::cuda_fail(e, "pack_dense_generic_kernel");
    return SBF_OK;
}
