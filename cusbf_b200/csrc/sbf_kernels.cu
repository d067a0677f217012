// sbf_kernels.cu -- sm_100a insert / query kernels of the Super Bloom engine.
//
// Reference path replaced: include/cusbf/detail/kernels.cuh:179-312 of
// tdortman/cuSBF (insert_sequence_kmers_kernel, contains_sequence_kmers_kernel
// and their dense-packed twins).  Results are bit-identical to it; the work
// decomposition is new:
//
//   * A persistent CTA walks tiles of 4096 consecutive windows.  Each tile's
//     input bytes are staged into shared memory by a 1D bulk async copy (TMA)
//     on an mbarrier, double-buffered so the next tile's copy overlaps the
//     current tile's hashing.  Only the 16-byte aligned interior goes through
//     the bulk copy; ragged edges are read with plain loads, so nothing
//     outside the caller's buffer is touched.
//   * Staged bytes are encoded with SWAR into 2-bit code words (16 bases per
//     32-bit word, earliest base in the top bits) plus invalid masks.
//   * Each thread owns a strip of 16 consecutive windows.  Every m-mer and
//     s-mer of the strip is one funnel shift of the code words, every
//     absolute position is hashed once, and the per-window minimizer is a
//     Gil-Werman sliding minimum (about 3 comparisons per window instead of
//     the reference's 16 multiplies).
//   * Insert merges consecutive windows that select the same shard (a
//     super-k-mer run) in registers and issues one red.or.b64 per shard word
//     per run.  Query loads each run's 32-byte shard once with a 256-bit
//     load and tests the findere rule (all k-s+1 s-mers present).
#include <cuda_runtime.h>

#include <cstdint>

#include "sbf_device.cuh"
#include "sbf_internal.h"

namespace sbf {

template <int K_, int S_, int M_, int H_>
struct Cfg {
    static constexpr int K = K_;
    static constexpr int S = S_;
    static constexpr int M = M_;
    static constexpr int H = H_;
    static constexpr int W = K - M + 1;  // m-mers per window
    static constexpr int F = K - S + 1;  // s-mers per window (findere span)
    static_assert(K >= 1 && K <= 32, "k must fit a 64-bit packed window");
    static_assert(M >= 1 && M <= 16 && M <= K, "m-mer must fit 32 bits");
    static_assert(S >= 1 && S <= K, "s must satisfy 1 <= s <= k");
    static_assert(H % 4 == 0 && H >= 4 && H <= 16, "hash count must be 4, 8, 12 or 16");
};

// ---------------------------------------------------------------------------
// Tile geometry and staging
// ---------------------------------------------------------------------------

struct TileGeom {
    uint64_t a;      // 16-byte aligned address of stage byte 0
    uint32_t off;    // stage offset of the tile's first input byte
    uint64_t lo, hi; // bulk-copied address range [lo, hi), empty when lo >= hi
    uint64_t r0, r1; // readable range of the input [r0, r1)
    uint32_t span;   // staged bytes
    int64_t b_lo;    // input byte index of stage offset `off`
    int64_t s0;      // symbol index of the tile's first grid position
};

template <bool kDense>
__device__ __forceinline__ TileGeom tile_geom(const TileParams& p, uint64_t tile) {
    TileGeom g;
    g.s0 = static_cast<int64_t>(tile) * kTileKmers + p.sym_base;
    uint32_t need;
    if constexpr (kDense) {
        // 2-bit symbols: symbol s sits at bit 2s of the byte stream.
        g.b_lo = g.s0 >= 0 ? g.s0 / 4 : -((-g.s0 + 3) / 4);
        need = (kCodeWords * 16 + 3) / 4 + 8;
    } else {
        g.b_lo = g.s0;
        need = kCodeWords * 16 + 4;
    }
    const uint64_t base = reinterpret_cast<uint64_t>(p.input);
    const uint64_t first = base + static_cast<uint64_t>(g.b_lo);  // wraps for b_lo < 0
    g.a = first & ~uint64_t{15};
    g.off = static_cast<uint32_t>(first & 15u);
    g.span = (g.off + need + 15u) & ~15u;
    g.r0 = base;
    g.r1 = base + p.input_bytes;
    const uint64_t in_lo = (base + 15u) & ~uint64_t{15};
    const uint64_t in_hi = g.r1 & ~uint64_t{15};
    // Signed comparisons: the stage window may start before the input.
    const int64_t a_s = static_cast<int64_t>(g.a - base);
    const int64_t lo_s = a_s > static_cast<int64_t>(in_lo - base) ? a_s
                                                                  : static_cast<int64_t>(in_lo - base);
    const int64_t hi_end = a_s + static_cast<int64_t>(g.span);
    const int64_t hi_s = hi_end < static_cast<int64_t>(in_hi - base)
                             ? hi_end
                             : static_cast<int64_t>(in_hi - base);
    g.lo = base + static_cast<uint64_t>(lo_s);
    g.hi = base + static_cast<uint64_t>(hi_s);
    if (hi_s <= lo_s) g.hi = g.lo;
    return g;
}

template <bool kDense>
__device__ __forceinline__ void issue_stage(const TileParams& p, uint64_t tile, uint8_t* buf,
                                            uint64_t* bar) {
    const TileGeom g = tile_geom<kDense>(p, tile);
    fence_proxy_async_smem();
    if (g.hi > g.lo) {
        const uint32_t bytes = static_cast<uint32_t>(g.hi - g.lo);
        mbar_arrive_expect_tx(bar, bytes);
        bulk_g2s(buf + (g.lo - g.a), reinterpret_cast<const void*>(g.lo), bytes, bar);
    } else {
        mbar_arrive(bar);
    }
}

// Plain loads of the readable bytes of the stage window that the bulk copy
// did not cover (at most 15 at each end of the input).
template <bool kDense>
__device__ __forceinline__ void fill_ragged(const TileParams& p, uint64_t tile, uint8_t* buf) {
    const TileGeom g = tile_geom<kDense>(p, tile);
    const int64_t base = static_cast<int64_t>(g.r0);
    const int64_t w0 = static_cast<int64_t>(g.a - g.r0);  // window start rel. to input
    const int64_t w1 = w0 + g.span;
    const int64_t in0 = 0, in1 = static_cast<int64_t>(p.input_bytes);
    const int64_t v0 = w0 > in0 ? w0 : in0;  // readable part of the window
    const int64_t v1 = w1 < in1 ? w1 : in1;
    if (v1 <= v0) return;
    const int64_t c0 = static_cast<int64_t>(g.lo) - base;
    const int64_t c1 = static_cast<int64_t>(g.hi) - base;
    // Head [v0, c0) and tail [c1, v1) when a bulk copy ran; otherwise all.
    int64_t h0 = v0, h1 = v1, t0 = 0, t1 = 0;
    if (c1 > c0) {
        h1 = c0 < v1 ? c0 : v1;
        t0 = c1 > v0 ? c1 : v0;
        t1 = v1;
    }
    const int tid = threadIdx.x;
    const int64_t nh = h1 > h0 ? h1 - h0 : 0;
    const int64_t nt = t1 > t0 ? t1 - t0 : 0;
    for (int64_t x = tid; x < nh + nt; x += kThreads) {
        const int64_t src = x < nh ? h0 + x : t0 + (x - nh);
        buf[src - w0] = p.input[src];
    }
}

// Encodes code word q (16 symbols from grid position 16q) of the staged tile.
template <bool kDense>
__device__ __forceinline__ void encode_word(const TileGeom& g, const uint8_t* buf, int q,
                                            uint32_t& code, uint32_t& inval) {
    const uint32_t* w32 = reinterpret_cast<const uint32_t*>(buf);
    if constexpr (kDense) {
        const int64_t sym_in_stage = g.s0 - 4 * g.b_lo;  // 0..3
        const uint32_t bitpos = 8u * g.off + 2u * static_cast<uint32_t>(sym_in_stage) + 32u * q;
        const uint32_t wi = bitpos >> 5;
        const uint32_t v = __funnelshift_r(w32[wi], w32[wi + 1], bitpos & 31u);
        code = dense16_to_code(v);
        inval = 0u;
    } else {
        const uint32_t bytepos = g.off + 16u * q;
        const uint32_t wi = bytepos >> 2;
        const uint32_t sh = (bytepos & 3u) * 8u;
        const uint32_t x0 = w32[wi], x1 = w32[wi + 1], x2 = w32[wi + 2], x3 = w32[wi + 3],
                       x4 = w32[wi + 4];
        encode16(__funnelshift_r(x0, x1, sh), __funnelshift_r(x1, x2, sh),
                 __funnelshift_r(x2, x3, sh), __funnelshift_r(x3, x4, sh), code, inval);
    }
}

// ---------------------------------------------------------------------------
// Strip computation: 16 windows per thread
// ---------------------------------------------------------------------------

template <class C>
struct Strip {
    uint32_t shard[kStrip];
    uint32_t vmask;  // bit j: window j is in range and holds only valid bases
};

// A[r]: the 16 bases starting at strip position r, earliest base in bits 31:30.
__device__ __forceinline__ uint32_t win16(uint32_t c0, uint32_t c1, uint32_t c2, int r) {
    return r < 16 ? __funnelshift_l(c1, c0, 2 * r) : __funnelshift_l(c2, c1, 2 * (r - 16));
}

template <class C>
__device__ __forceinline__ uint64_t smer_at(uint32_t c0, uint32_t c1, uint32_t c2, int r) {
    if constexpr (C::S > 16) {
        const uint64_t hi = win16(c0, c1, c2, r) >> (2 * (32 - C::S));
        return (hi << 32) | win16(c0, c1, c2, r + C::S - 16);
    } else {
        return win16(c0, c1, c2, r) >> (2 * (16 - C::S));
    }
}

template <class C>
__device__ __forceinline__ void strip_shards(uint32_t c0, uint32_t c1, uint32_t c2,
                                             uint32_t shard_mask, uint32_t* shard) {
    constexpr int W = C::W;
    constexpr int NP = kStrip + W - 1;  // m-mer positions used by the strip
    if constexpr (W == 16) {
        // Gil-Werman: suffix minima of block [0,16), running prefix minima
        // of block [16, 31); window j = min(suffix[j], prefix[j-1]).
        uint64_t suf[16];
        suf[15] = mmer_hash(win16(c0, c1, c2, 15) >> (2 * (16 - C::M)));
#pragma unroll
        for (int r = 14; r >= 0; --r)
            suf[r] = min64(mmer_hash(win16(c0, c1, c2, r) >> (2 * (16 - C::M))), suf[r + 1]);
        shard[0] = static_cast<uint32_t>(suf[0]) & shard_mask;
        uint64_t pre = ~uint64_t{0};
#pragma unroll
        for (int j = 1; j < kStrip; ++j) {
            pre = min64(pre, mmer_hash(win16(c0, c1, c2, 15 + j) >> (2 * (16 - C::M))));
            shard[j] = static_cast<uint32_t>(min64(suf[j], pre)) & shard_mask;
        }
    } else {
        uint64_t mh[NP];
#pragma unroll
        for (int r = 0; r < NP; ++r) mh[r] = mmer_hash(win16(c0, c1, c2, r) >> (2 * (16 - C::M)));
#pragma unroll
        for (int j = 0; j < kStrip; ++j) {
            uint64_t v = mh[j];
#pragma unroll
            for (int o = 1; o < W; ++o) v = min64(v, mh[j + o]);
            shard[j] = static_cast<uint32_t>(v) & shard_mask;
        }
    }
}

// Valid-window mask of the strip: window j holds K valid bases and lies in
// [0, n_kmers).
template <class C>
__device__ __forceinline__ uint32_t strip_valid(uint32_t i0, uint32_t i1, uint32_t i2,
                                                int64_t first_kmer, uint64_t n_kmers) {
    uint32_t vmask = 0xFFFFu;
    const uint64_t inv = static_cast<uint64_t>(i0) | (static_cast<uint64_t>(i1) << 16) |
                         (static_cast<uint64_t>(i2) << 32);
    constexpr uint64_t kWin = (C::K >= 64) ? ~uint64_t{0} : ((uint64_t{1} << C::K) - 1);
    if (inv & ((uint64_t{1} << (15 + C::K)) - 1)) {
#pragma unroll
        for (int j = 0; j < kStrip; ++j)
            if ((inv >> j) & kWin) vmask &= ~(1u << j);
    }
    if (first_kmer < 0 || first_kmer + kStrip > static_cast<int64_t>(n_kmers)) {
#pragma unroll
        for (int j = 0; j < kStrip; ++j) {
            const int64_t i = first_kmer + j;
            if (i < 0 || i >= static_cast<int64_t>(n_kmers)) vmask &= ~(1u << j);
        }
    }
    return vmask;
}

// Four word masks of the s-mer at strip position r.
template <class C>
__device__ __forceinline__ void smer_masks(uint32_t c0, uint32_t c1, uint32_t c2, int r,
                                           uint64_t m[4]) {
    const uint64_t h = smer_hash(smer_at<C>(c0, c1, c2, r));
    m[0] = m[1] = m[2] = m[3] = 0;
#pragma unroll
    for (int j = 0; j < C::H; ++j) m[j & 3] |= uint64_t{1} << bit_address<C::H>(h, j);
}

// True when every bit of the s-mer at strip position r is set in w0..w3.
template <class C>
__device__ __forceinline__ uint32_t smer_present(uint64_t h, uint64_t w0, uint64_t w1,
                                                 uint64_t w2, uint64_t w3) {
    uint64_t acc = ~uint64_t{0};
#pragma unroll
    for (int j = 0; j < C::H; ++j) {
        const uint64_t w = (j & 3) == 0 ? w0 : (j & 3) == 1 ? w1 : (j & 3) == 2 ? w2 : w3;
        acc &= w >> bit_address<C::H>(h, j);
    }
    return static_cast<uint32_t>(acc) & 1u;
}

template <class C>
__device__ __forceinline__ void insert_strip(uint32_t c0, uint32_t c1, uint32_t c2,
                                             const uint32_t* shard, uint32_t vmask,
                                             uint64_t* words) {
    constexpr int F = C::F;
    constexpr int NP = kStrip + F - 1;
    uint64_t pm[NP][4];
#pragma unroll
    for (int r = 0; r < NP; ++r) smer_masks<C>(c0, c1, c2, r, pm[r]);
    uint64_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
    for (int j = 0; j < kStrip; ++j) {
        uint64_t t0 = pm[j][0], t1 = pm[j][1], t2 = pm[j][2], t3 = pm[j][3];
#pragma unroll
        for (int o = 1; o < F; ++o) {
            t0 |= pm[j + o][0];
            t1 |= pm[j + o][1];
            t2 |= pm[j + o][2];
            t3 |= pm[j + o][3];
        }
        const bool valid = (vmask >> j) & 1u;
        const bool cont = j > 0 && ((vmask >> (j - 1)) & 1u) && shard[j] == shard[j - 1];
        a0 = cont ? (a0 | t0) : t0;
        a1 = cont ? (a1 | t1) : t1;
        a2 = cont ? (a2 | t2) : t2;
        a3 = cont ? (a3 | t3) : t3;
        const bool next_cont =
            j + 1 < kStrip && ((vmask >> (j + 1)) & 1u) && shard[j + 1] == shard[j];
        if (valid && !next_cont) {
            uint64_t* dst = words + static_cast<uint64_t>(shard[j]) * 4;
            red_or(dst + 0, a0);
            red_or(dst + 1, a1);
            red_or(dst + 2, a2);
            red_or(dst + 3, a3);
        }
    }
}

template <class C>
__device__ __forceinline__ uint32_t query_strip(uint32_t c0, uint32_t c1, uint32_t c2,
                                                const uint32_t* shard, uint32_t vmask,
                                                const uint64_t* words) {
    constexpr int F = C::F;
    constexpr int NP = kStrip + F - 1;
    uint64_t h[NP];
#pragma unroll
    for (int r = 0; r < NP; ++r) h[r] = smer_hash(smer_at<C>(c0, c1, c2, r));
    uint32_t result = 0;
    uint64_t w0 = 0, w1 = 0, w2 = 0, w3 = 0;
    bool have = false;
    uint32_t cur = 0;
#pragma unroll
    for (int j = 0; j < kStrip; ++j) {
        const bool valid = (vmask >> j) & 1u;
        const bool head = valid && (!have || shard[j] != cur);
        if (head) {
            load_shard(words + static_cast<uint64_t>(shard[j]) * 4, w0, w1, w2, w3);
            cur = shard[j];
            have = true;
        }
        uint32_t present = valid ? 1u : 0u;
#pragma unroll
        for (int o = 0; o < F; ++o) present &= smer_present<C>(h[j + o], w0, w1, w2, w3);
        result |= present << j;
    }
    return result;
}

__device__ __forceinline__ uint32_t spread4(uint32_t nib) {
    return (nib * 0x00204081u) & 0x01010101u;
}

// ---------------------------------------------------------------------------
// The tile kernel
// ---------------------------------------------------------------------------

template <class C, bool kQuery, bool kDense>
__global__ void __launch_bounds__(kThreads) tile_kernel(TileParams p) {
    __shared__ alignas(128) uint8_t stage[2][kStageBytes];
    __shared__ uint32_t code[kCodeWords + 2];
    __shared__ uint32_t inval[kCodeWords + 2];
    __shared__ alignas(8) uint64_t bars[2];

    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
    }
    __syncthreads();

    const uint64_t stride = gridDim.x;
    uint64_t tile = blockIdx.x;
    if (tid == 0) {
        if (tile < p.n_tiles) issue_stage<kDense>(p, tile, stage[0], &bars[0]);
        if (tile + stride < p.n_tiles) issue_stage<kDense>(p, tile + stride, stage[1], &bars[1]);
    }
    uint32_t it = 0;
    for (; tile < p.n_tiles; tile += stride, ++it) {
        const int b = it & 1;
        const uint32_t parity = (it >> 1) & 1u;
        const bool ok = mbar_wait_bounded(&bars[b], parity);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(p.err, kDevErrStageTimeout);
            // Give the other buffer's copy (if any) a bounded chance to land
            // before the CTA's shared memory is released.
            if (tile + stride < p.n_tiles) (void)mbar_wait_bounded(&bars[b ^ 1], parity);
            return;
        }
        fill_ragged<kDense>(p, tile, stage[b]);
        __syncthreads();
        const TileGeom g = tile_geom<kDense>(p, tile);
        for (int q = tid; q < kCodeWords; q += kThreads) {
            uint32_t cw, iv;
            encode_word<kDense>(g, stage[b], q, cw, iv);
            code[q] = cw;
            inval[q] = iv;
        }
        __syncthreads();
        if (tid == 0 && tile + 2 * stride < p.n_tiles)
            issue_stage<kDense>(p, tile + 2 * stride, stage[b], &bars[b]);

        const uint32_t c0 = code[tid], c1 = code[tid + 1], c2 = code[tid + 2];
        const int64_t first_kmer = g.s0 + static_cast<int64_t>(tid) * kStrip;
        const uint32_t vmask =
            strip_valid<C>(inval[tid], inval[tid + 1], inval[tid + 2], first_kmer, p.n_kmers);
        uint32_t shard[kStrip];
        strip_shards<C>(c0, c1, c2, p.shard_mask, shard);
        if constexpr (kQuery) {
            const uint32_t res = query_strip<C>(c0, c1, c2, shard, vmask, p.words);
            // Windows outside [0, n_kmers) are not written; the rest get 0/1.
            if (first_kmer >= 0 && first_kmer + kStrip <= static_cast<int64_t>(p.n_kmers)) {
                uint4 v;
                v.x = spread4(res & 0xFu);
                v.y = spread4((res >> 4) & 0xFu);
                v.z = spread4((res >> 8) & 0xFu);
                v.w = spread4((res >> 12) & 0xFu);
                *reinterpret_cast<uint4*>(p.out + first_kmer) = v;
            } else {
#pragma unroll
                for (int j = 0; j < kStrip; ++j) {
                    const int64_t i = first_kmer + j;
                    if (i >= 0 && i < static_cast<int64_t>(p.n_kmers))
                        p.out[i] = static_cast<uint8_t>((res >> j) & 1u);
                }
            }
        } else {
            if (vmask) insert_strip<C>(c0, c1, c2, shard, vmask, p.words);
        }
    }
}

// ---------------------------------------------------------------------------
// Auxiliary kernels
// ---------------------------------------------------------------------------

// Dense packing: 32 symbols per word, symbol t at bits [2t, 2t+2), invalid
// bytes stored as their low two code bits (include/cusbf/dense_packed.hpp:26-50).
__global__ void pack_dense_kernel(const uint8_t* seq, uint64_t num_symbols, uint64_t* words) {
    const uint64_t w = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t n_words = (num_symbols + 31) / 32;
    if (w >= n_words) return;
    const uint64_t first = w * 32;
    uint64_t out = 0;
    for (int t = 0; t < 32; ++t) {
        const uint64_t s = first + t;
        if (s >= num_symbols) break;
        const uint8_t b = seq[s];
        const uint8_t upper = b & 0xDFu;
        const bool valid = upper == 'A' || upper == 'C' || upper == 'G' || upper == 'T';
        const uint64_t code = valid ? ((b >> 1) & 3u) : 3u;
        out |= code << (2 * t);
    }
    words[w] = out;
}

__global__ void popcount_kernel(const uint64_t* words, uint64_t n, unsigned long long* out) {
    unsigned long long local = 0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        local += __popcll(words[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xFFFFFFFFu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(out, local);
}

cudaError_t launch_pack_dense(const uint8_t* seq, uint64_t num_symbols, uint64_t* words,
                              cudaStream_t stream) {
    const uint64_t n_words = (num_symbols + 31) / 32;
    if (n_words == 0) return cudaSuccess;
    pack_dense_kernel<<<static_cast<unsigned>((n_words + 255) / 256), 256, 0, stream>>>(
        seq, num_symbols, words);
    return cudaGetLastError();
}

cudaError_t launch_popcount(const uint64_t* words, uint64_t n_words, unsigned long long* out,
                            cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    if (n_words == 0) return cudaSuccess;
    uint64_t blocks = (n_words + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    popcount_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(words, n_words, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Compiled configurations
// ---------------------------------------------------------------------------

template <int K, int S, int M, int H>
constexpr KernelSet make_set() {
    using C = Cfg<K, S, M, H>;
    return KernelSet{K,
                     S,
                     M,
                     H,
                     &tile_kernel<C, false, false>,
                     &tile_kernel<C, true, false>,
                     &tile_kernel<C, false, true>,
                     &tile_kernel<C, true, true>};
}

static const KernelSet kSets[] = {
    make_set<31, 28, 16, 4>(),  // the graded configuration
    make_set<31, 30, 16, 4>(),  make_set<31, 31, 16, 4>(), make_set<31, 28, 16, 8>(),
    make_set<31, 28, 16, 16>(), make_set<21, 19, 11, 4>(), make_set<5, 4, 3, 4>(),
    make_set<3, 2, 2, 4>(),
};

const KernelSet* find_kernels(int k, int s, int m, int h) {
    for (const KernelSet& ks : kSets)
        if (ks.k == k && ks.s == s && ks.m == m && ks.h == h) return &ks;
    return nullptr;
}

}  // namespace sbf
