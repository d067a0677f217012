// sbf_generic.cuh -- runtime-parameterised insert / query kernels for every
// configuration that has no specialised tile kernel: any k, s, m and hash
// count the reference's Config accepts (config.cuh:28-118), and the protein
// and DNA-triplet alphabets (Alphabet.cuh:150-220).
//
// Each thread owns a strip of 32 consecutive windows.  The strip's k-mer is
// packed MSB-first and slid one symbol per window
// (detail/sequence_kmer.cuh:75-90); every window takes the minimum of its
// m-mer hashes (minimizer_hash64, hashutil.cuh:207-209) for the shard and the
// union of its s-mers' bit masks (hash64, hashutil.cuh:192-196;
// sectorizedBitAddress, detail/filter_impl.cuh:37-77), exactly as the
// reference evaluates one window.  Inserts OR a run of windows that select
// the same shard into one set of four atomics; queries reuse the loaded
// shard while the run continues.  A window is valid when none of its symbols
// is invalid (dense input is always valid) and, for ragged launches, when
// its bytes lie inside one record.
//
// The kernels take the same TileParams and launch shape as the tile kernels
// (with no dynamic shared memory, so more CTAs fit an SM), so every caller --
// plain launches, host pipelines, ragged batches, the server -- runs them
// unchanged.
//
// Device code only: compiled into the library (RuntimeGen) by sbf_generic.cu,
// and for one configuration at run time (FixedGen) by sbf_jit.cpp.
#pragma once

#include "sbf_device.cuh"
#include "sbf_flush.cuh"
#include "sbf_internal.h"

namespace sbf {

// Alphabet ids (SBF_ALPHABET_* of the C ABI).
constexpr uint32_t kAlphabetDna = 0, kAlphabetTriplet = 1, kAlphabetProtein = 2;

constexpr uint8_t kInvalid = 0xFFu;

__device__ __forceinline__ uint8_t dna_code(uint8_t b) {
    const uint8_t u = b & 0xDFu;
    const bool ok = u == 'A' || u == 'C' || u == 'G' || u == 'T';
    return ok ? static_cast<uint8_t>((b >> 1) & 3u) : kInvalid;
}

// Alphabet::encode (Alphabet.cuh:132-141, 160-175, 200-215).
__device__ __forceinline__ uint8_t encode_symbol(const GenericCfg& c, const uint8_t* p) {
    if (c.alphabet == kAlphabetProtein) {
        const uint8_t idx = static_cast<uint8_t>((p[0] & 0xDFu) - 'A');
        return idx < 26 ? idx : kInvalid;
    }
    if (c.alphabet == kAlphabetTriplet) {
        const uint8_t a = dna_code(p[0]), b = dna_code(p[1]), d = dna_code(p[2]);
        if (a == kInvalid || b == kInvalid || d == kInvalid) return kInvalid;
        return static_cast<uint8_t>((a << 4) | (b << 2) | d);
    }
    return dna_code(p[0]);
}

template <bool kDense>
__device__ __forceinline__ uint8_t symbol_at(const TileParams& p, uint64_t t) {
    const GenericCfg& c = p.gen;
    if constexpr (kDense) {
        // 64 / bits symbols per word, symbol t at bit (t % per_word) * bits
        // (detail/dense_packed.cuh:44-60).
        const uint32_t per_word = 64u / c.bits;
        const uint64_t w = reinterpret_cast<const uint64_t*>(p.input)[t / per_word];
        return static_cast<uint8_t>((w >> ((t % per_word) * c.bits)) & ((1u << c.bits) - 1u));
    } else {
        return encode_symbol(c, p.input + t * c.width);
    }
}

__device__ __forceinline__ uint64_t low_mask(uint32_t bits) {
    return bits >= 64 ? ~uint64_t{0} : ((uint64_t{1} << bits) - 1);
}

// Bit j of an s-mer hash (detail/filter_impl.cuh:37-48).
__device__ __forceinline__ uint32_t bit_address(uint32_t h, uint32_t j, uint64_t x) {
    const uint32_t slice = 64u / h;
    if (slice >= 6) return static_cast<uint32_t>((x >> (slice * j)) & 63u);
    return static_cast<uint32_t>((x * salt(static_cast<int>(j))) >> 58);
}

// Shard and the four word masks of one packed k-mer.
__device__ __forceinline__ uint32_t eval_kmer(const GenericCfg& c, uint32_t shard_mask,
                                              uint64_t km, uint64_t masks[4]) {
    const uint64_t mm_mask = low_mask(c.m * c.bits);
    uint64_t minh = ~uint64_t{0};
#pragma unroll
    for (uint32_t o = 0; o + c.m <= c.k; ++o) {
        const uint64_t mm = (km >> (c.bits * (c.k - o - c.m))) & mm_mask;
        const uint64_t hh = mm * kMinimizerMul;
        minh = hh < minh ? hh : minh;
    }
    masks[0] = masks[1] = masks[2] = masks[3] = 0;
    const uint64_t sm_mask = low_mask(c.s * c.bits);
#pragma unroll
    for (uint32_t o = 0; o + c.s <= c.k; ++o) {
        uint64_t x = ((km >> (c.bits * (c.k - o - c.s))) & sm_mask) * kSmerMul;
        x ^= x >> 33;
#pragma unroll
        for (uint32_t j = 0; j < c.h; ++j) masks[j & 3] |= uint64_t{1} << bit_address(c.h, j, x);
    }
    return static_cast<uint32_t>(minh) & shard_mask;
}

// The configuration comes from the launch (RuntimeGen, one build for every
// configuration) or from template constants (FixedGen, compiled at run time
// for one configuration so loops unroll and shifts are constants).
// FixedGen inserts flush each run with one 32-byte bulk OR-reduction from
// the flush ring in the launch's dynamic shared memory; RuntimeGen launches
// have none and use four 8-byte atomics.
struct RuntimeGen {
    static constexpr bool kBulkFlush = false;
    __device__ __forceinline__ static GenericCfg get(const TileParams& p) { return p.gen; }
};
template <int K, int S, int M, int H, int Bits, int Width, int Alphabet>
struct FixedGen {
    static constexpr bool kBulkFlush = true;
    static constexpr int kK = K, kS = S, kM = M, kH = H, kBits = Bits;
    __device__ __forceinline__ static GenericCfg get(const TileParams&) {
        return GenericCfg{K, S, M, H, Bits, Width, Alphabet};
    }
};

// The four word masks of one s-mer value (hash64, hashutil.cuh:192-196;
// sectorizedBitAddress, detail/filter_impl.cuh:37-77).
__device__ __forceinline__ void smer_value_masks(uint32_t h, uint64_t sm, uint64_t m[4]) {
    uint64_t x = sm * kSmerMul;
    x ^= x >> 33;
    m[0] = m[1] = m[2] = m[3] = 0;
#pragma unroll
    for (uint32_t j = 0; j < h; ++j) m[j & 3] |= uint64_t{1} << bit_address(h, j, x);
}

template <class G, bool kQuery, bool kDense, bool kRagged>
__global__ void __launch_bounds__(kThreads) generic_kernel(TileParams p) {
    const GenericCfg c = G::get(p);
    extern __shared__ __align__(16) uint64_t flush_slots[];
    FlushRing ring{flush_slots + 4 * threadIdx.x, 0u};
    (void)ring;
    const uint64_t n = p.n_kmers;
    const uint64_t n_strips = (n + kStrip - 1) / kStrip;
    const uint64_t km_mask = low_mask(c.k * c.bits);
    const uint64_t sym_mask = (uint64_t{1} << c.bits) - 1;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    unsigned long long n_valid = 0, n_pos = 0;
    for (uint64_t st = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; st < n_strips;
         st += stride) {
        const uint64_t w0 = st * kStrip;
        const uint64_t w_end = w0 + kStrip < n ? w0 + kStrip : n;
        // Prime the first k-1 symbols of window w0.
        uint64_t km = 0;
        int64_t last_inv = -1;  // latest invalid symbol index seen
        for (uint32_t j = 0; j + 1 < c.k; ++j) {
            const uint64_t t = w0 + j;
            const uint8_t e = symbol_at<kDense>(p, t);
            if (!kDense && e == kInvalid) last_inv = static_cast<int64_t>(t);
            km = ((km << c.bits) | (e & sym_mask)) & km_mask;
        }
        // Ragged: the record holding the current window's first byte
        // (window w covers bytes [w * width, (w + k) * width)).
        uint64_t r = 0;
        if constexpr (kRagged) {
            uint64_t lo = 0, hi = p.n_ranges;
            while (lo < hi) {
                const uint64_t mid = (lo + hi) >> 1;
                if (p.ranges[mid].offset + p.ranges[mid].bytes > w0 * c.width)
                    hi = mid;
                else
                    lo = mid + 1;
            }
            r = lo;
        }
        bool in_run = false;
        uint32_t run_shard = 0;
        uint64_t acc[4] = {0, 0, 0, 0};   // insert: the run's merged masks
        uint64_t words[4] = {0, 0, 0, 0};  // query: the run's shard words
        uint32_t hits = 0;
        uint64_t rec_cur = ~uint64_t{0};
        unsigned long long rv = 0, rp = 0;  // the current record's tallies
        auto flush_record = [&]() {
            if (rec_cur != ~uint64_t{0} && (rv | rp)) {
                const uint64_t at = rec_cur << p.rec_shift;
                if (rv) atomicAdd(p.rec_valid + at, rv);
                if (rp) atomicAdd(p.rec_pos + at, rp);
            }
            rv = rp = 0;
        };
        auto flush_run_now = [&]() {
            if (!kQuery && in_run) {
                if constexpr (G::kBulkFlush) {
                    flush_run(p.words, run_shard, acc, ring);
                } else {
                    uint64_t* dst = p.words + static_cast<uint64_t>(run_shard) * 4;
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        if (acc[i]) atomicOr(reinterpret_cast<unsigned long long*>(dst + i), acc[i]);
                }
            }
        };
        // Window w: its next symbol enters km; returns whether it is valid.
        auto advance = [&](uint64_t w) -> bool {
            const uint64_t t = w + c.k - 1;
            const uint8_t e = symbol_at<kDense>(p, t);
            if (!kDense && e == kInvalid) last_inv = static_cast<int64_t>(t);
            km = ((km << c.bits) | (e & sym_mask)) & km_mask;
            bool valid = last_inv < static_cast<int64_t>(w);
            if constexpr (kRagged) {
                const uint64_t b0 = w * c.width;
                while (r < p.n_ranges && p.ranges[r].offset + p.ranges[r].bytes <= b0) ++r;
                valid = valid && r < p.n_ranges && p.ranges[r].offset <= b0 &&
                        (w + c.k) * c.width <= p.ranges[r].offset + p.ranges[r].bytes;
            }
            return valid;
        };
        // A valid window w with its shard and word masks: query test or run
        // merge, record tallies; `hit` is written for every window.
        auto apply = [&](uint64_t w, bool valid, uint32_t shard, const uint64_t m[4]) {
            bool hit = false;
            if (valid) {
                if constexpr (kQuery) {
                    if (!in_run || shard != run_shard) {
                        load_shard(p.words + static_cast<uint64_t>(shard) * 4, words[0], words[1],
                                   words[2], words[3]);
                        run_shard = shard;
                        in_run = true;
                    }
                    hit = ((words[0] & m[0]) == m[0]) && ((words[1] & m[1]) == m[1]) &&
                          ((words[2] & m[2]) == m[2]) && ((words[3] & m[3]) == m[3]);
                } else {
                    if (!in_run || shard != run_shard) {
                        flush_run_now();
                        run_shard = shard;
                        in_run = true;
                        acc[0] = acc[1] = acc[2] = acc[3] = 0;
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i) acc[i] |= m[i];
                }
                if constexpr (kRagged) {
                    ++n_valid;
                    n_pos += hit;
                    if (p.rec_valid) {
                        if (r != rec_cur) {
                            flush_record();
                            rec_cur = r;
                        }
                        ++rv;
                        rp += hit;
                    }
                }
            }
            if constexpr (kQuery) {
                if (p.out) p.out[w] = hit ? 1 : 0;
                hits |= static_cast<uint32_t>(hit) << (w - w0);
            }
        };
        if constexpr (G::kBulkFlush && !kQuery) {
            // Inserts with configuration constants: each window hashes only
            // its newest m-mer and s-mer, kept in rings of the window's W
            // m-mer hashes and F s-mer masks (slot x % W holds the m-mer
            // starting at symbol w0 + x).  The strip is unrolled, so ring
            // slots are registers.  (Protein <12,10,6,4>: insert 72.8 -> 76.9
            // G windows/s; the same form made the query 16% slower, so
            // queries evaluate each window whole.)
            constexpr int kK = G::kK, kM = G::kM, kS = G::kS, kBits = G::kBits;
            constexpr int W = kK - kM + 1, F = kK - kS + 1;
            const uint64_t mm_mask = low_mask(kM * kBits);
            const uint64_t sm_mask = low_mask(kS * kBits);
            uint64_t mh[W], sm[F][4];
#pragma unroll
            for (int o = 0; o < W - 1; ++o)
                mh[o] = ((km >> (kBits * (kK - 1 - o - kM))) & mm_mask) * kMinimizerMul;
#pragma unroll
            for (int o = 0; o < F - 1; ++o)
                smer_value_masks(G::kH, (km >> (kBits * (kK - 1 - o - kS))) & sm_mask, sm[o]);
#pragma unroll
            for (int j = 0; j < kStrip; ++j) {
                const uint64_t w = w0 + j;
                if (w >= w_end) break;
                const bool valid = advance(w);
                mh[(j + W - 1) % W] = (km & mm_mask) * kMinimizerMul;
                smer_value_masks(G::kH, km & sm_mask, sm[(j + F - 1) % F]);
                uint64_t m[4] = {0, 0, 0, 0};
                uint32_t shard = 0;
                if (valid) {
                    uint64_t minh = mh[0];
#pragma unroll
                    for (int o = 1; o < W; ++o) minh = mh[o] < minh ? mh[o] : minh;
                    shard = static_cast<uint32_t>(minh) & p.shard_mask;
#pragma unroll
                    for (int o = 0; o < F; ++o) {
#pragma unroll
                        for (int q = 0; q < 4; ++q) m[q] |= sm[o][q];
                    }
                }
                apply(w, valid, shard, m);
            }
        } else {
            for (uint64_t w = w0; w < w_end; ++w) {
                const bool valid = advance(w);
                uint64_t m[4] = {0, 0, 0, 0};
                const uint32_t shard = valid ? eval_kmer(c, p.shard_mask, km, m) : 0u;
                apply(w, valid, shard, m);
            }
        }
        flush_run_now();
        if constexpr (kRagged) flush_record();
        if constexpr (kQuery) {
            if (p.out_bits) p.out_bits[w0 / kStrip] = hits;
        }
    }
    if constexpr (!kQuery && G::kBulkFlush) flush_ring_drain();
    if constexpr (kRagged) {
        if (p.counts) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                n_valid += __shfl_down_sync(0xFFFFFFFFu, n_valid, o);
                n_pos += __shfl_down_sync(0xFFFFFFFFu, n_pos, o);
            }
            if ((threadIdx.x & 31) == 0) {
                if (n_valid) atomicAdd(p.counts, n_valid);
                if (n_pos) atomicAdd(p.counts + 1, n_pos);
            }
        }
    }
}

}  // namespace sbf
