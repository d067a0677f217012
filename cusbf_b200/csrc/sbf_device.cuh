// sbf_device.cuh -- device building blocks of the Super Bloom engine (sm_100a).
//
// Semantics follow the reference cuSBF (tdortman/cuSBF); the arithmetic is
// re-derived for a strip-per-thread sliding formulation:
//   * DNA encode A0 C1 T2 G3, case-insensitive      include/cusbf/Alphabet.cuh:132-141
//   * m-mer hash  x * 0x9E3779B97F4A7C15            include/cusbf/hashutil.cuh:207-209
//   * s-mer hash  x * 0x9e3779b97f4a7c15 ^ (>> 33)  include/cusbf/hashutil.cuh:192-196
//   * bit address (h >> (64/H)*j) & 63 or (h * salt_j) >> 58
//                                                   include/cusbf/detail/filter_impl.cuh:37-48
//   * salts                                         include/cusbf/detail/filter_common.cuh:30-94
// The k-mer of window i is packed MSB-first (earliest base in the highest
// bits, include/cusbf/detail/sequence_kmer.cuh:75-82), so the m-mer / s-mer at
// offset o of window i equals the m-mer / s-mer starting at absolute base
// i + o.  Hashing each absolute position once and taking a sliding minimum
// therefore reproduces the per-window values bit for bit.
#pragma once

#ifndef __CUDACC_RTC__
#include <cstdint>
#endif

namespace sbf {

constexpr uint64_t kMinimizerMul = 0x9E3779B97F4A7C15ULL;
constexpr uint64_t kSmerMul = 0x9e3779b97f4a7c15ULL;

__device__ __forceinline__ uint64_t salt(int j) {
    // Multiplicative salts for hash counts whose 64/H slice is narrower than
    // six bits (H = 12, 16); values from include/cusbf/detail/filter_common.cuh:30-94.
    switch (j) {
        case 0: return 0x9E3779B97F4A7C15ULL;
        case 1: return 0xC2B2AE3D27D4EB4FULL;
        case 2: return 0x165667B19E3779F9ULL;
        case 3: return 0x85EBCA77C2B2AE63ULL;
        case 4: return 0x27D4EB2F165667C5ULL;
        case 5: return 0x94D049BB133111EFULL;
        case 6: return 0xBF58476D1CE4E5B9ULL;
        case 7: return 0xD6E8FEB86659FD93ULL;
        case 8: return 0xA0761D6478BD642FULL;
        case 9: return 0xE7037ED1A0B428DBULL;
        case 10: return 0x8EBC6AF09C88C6E3ULL;
        case 11: return 0x589965CC75374CC3ULL;
        case 12: return 0x1D8E4E27C47D124FULL;
        case 13: return 0xEB449C93FBBEA6B5ULL;
        case 14: return 0xDB4F0B9175AE2165ULL;
        default: return 0xBBE056FDADE14B91ULL;
    }
}

// ------------------------------------------------------------------------
// Encoding: 16 ASCII bases (four little-endian words) -> one 32-bit code word
// (earliest base in bits 31:30) and a 16-bit invalid mask (bit r = base r).
// ------------------------------------------------------------------------

// Packs the 2-bit codes held in the four bytes of `c` into the top byte,
// earliest byte first: byte r lands at bits (31-2r):(30-2r).
__device__ __forceinline__ uint32_t pack4_top(uint32_t c) { return c * 0x40100401u; }

__device__ __forceinline__ uint32_t invalid4(uint32_t v, uint32_t c) {
    // Expected upper-case letter for each byte's code: table A C T G indexed
    // by the code; a byte is valid exactly when (byte & 0xDF) equals it.
    const uint32_t s = c | (c >> 4);
    const uint32_t e_lo = __byte_perm(0x47544341u, 0u, s);
    const uint32_t e_hi = __byte_perm(0x47544341u, 0u, s >> 16);
    const uint32_t expect = __byte_perm(e_lo, e_hi, 0x5410u);
    return (v & 0xDFDFDFDFu) ^ expect;  // non-zero byte <=> invalid base
}

__device__ __forceinline__ uint32_t nonzero_bytes_to_bits(uint32_t d) {
    const uint32_t nz = (((d & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | d) & 0x80808080u;
    return ((nz >> 7) * 0x10204080u) >> 28;
}

__device__ __forceinline__ void encode16(uint32_t v0, uint32_t v1, uint32_t v2, uint32_t v3,
                                         uint32_t& code, uint32_t& inval) {
    const uint32_t c0 = (v0 >> 1) & 0x03030303u;
    const uint32_t c1 = (v1 >> 1) & 0x03030303u;
    const uint32_t c2 = (v2 >> 1) & 0x03030303u;
    const uint32_t c3 = (v3 >> 1) & 0x03030303u;
    const uint32_t lo = __byte_perm(pack4_top(c3), pack4_top(c2), 0x0073u);
    const uint32_t hi = __byte_perm(pack4_top(c1), pack4_top(c0), 0x0073u);
    code = __byte_perm(lo, hi, 0x5410u);
    const uint32_t d0 = invalid4(v0, c0);
    const uint32_t d1 = invalid4(v1, c1);
    const uint32_t d2 = invalid4(v2, c2);
    const uint32_t d3 = invalid4(v3, c3);
    if ((d0 | d1 | d2 | d3) == 0u) {
        inval = 0u;
    } else {
        inval = nonzero_bytes_to_bits(d0) | (nonzero_bytes_to_bits(d1) << 4) |
                (nonzero_bytes_to_bits(d2) << 8) | (nonzero_bytes_to_bits(d3) << 12);
    }
}

// 16 dense-packed symbols (LSB-first, 2 bits each) -> MSB-first code word.
__device__ __forceinline__ uint32_t dense16_to_code(uint32_t v) {
    const uint32_t r = __brev(v);
    return ((r >> 1) & 0x55555555u) | ((r & 0x55555555u) << 1);
}

// ------------------------------------------------------------------------
// Hashes
// ------------------------------------------------------------------------

__device__ __forceinline__ uint64_t mmer_hash(uint32_t mmer) {
    return static_cast<uint64_t>(mmer) * kMinimizerMul;
}

// m-mers longer than 16 bases.
__device__ __forceinline__ uint64_t mmer_hash(uint64_t mmer) { return mmer * kMinimizerMul; }

__device__ __forceinline__ uint64_t smer_hash(uint64_t smer) {
    uint64_t h = smer * kSmerMul;
    return h ^ (h >> 33);
}

__device__ __forceinline__ uint64_t min64(uint64_t a, uint64_t b) { return a < b ? a : b; }

template <int H>
__device__ __forceinline__ uint32_t bit_address(uint64_t h, int j) {
    constexpr int kSlice = 64 / H;
    if constexpr (kSlice >= 6) {
        return static_cast<uint32_t>((h >> (kSlice * j)) & 63u);
    } else {
        return static_cast<uint32_t>((h * salt(j)) >> 58);
    }
}

// ------------------------------------------------------------------------
// PTX wrappers: mbarrier + 1D bulk async copy (TMA) + vector loads / reds
// ------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_addr(bar)),
        "r"(bytes)
        : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for `parity` with a bound of roughly two seconds of SM clock; returns
// false on time-out instead of spinning forever.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    const long long start = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - start > (1LL << 32)) return false;
    }
    return true;
}

__device__ __forceinline__ void bulk_g2s(void* smem_dst, const void* gmem_src, uint32_t bytes,
                                         uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void load_shard(const uint64_t* p, uint64_t& w0, uint64_t& w1,
                                           uint64_t& w2, uint64_t& w3) {
    // One 32-byte sector per shard, read with a single 256-bit load; an L2
    // miss fills 64 bytes (.L2::64B) instead of 128.
    asm volatile("ld.global.nc.L2::64B.v4.u64 {%0, %1, %2, %3}, [%4];"
                 : "=l"(w0), "=l"(w1), "=l"(w2), "=l"(w3)
                 : "l"(p));
}

__device__ __forceinline__ void red_or(uint64_t* p, uint64_t v) {
    asm volatile("red.relaxed.gpu.global.or.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

}  // namespace sbf
