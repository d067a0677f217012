// sbf_tile.cuh -- sm_100a insert / query tile kernels of the Super Bloom engine
// (device code only: compiled into the library for the common configurations
// by sbf_kernels.cu, and for any other DNA configuration at run time by
// sbf_jit.cpp).
//
// Reference path replaced: include/cusbf/detail/kernels.cuh:179-312 of
// tdortman/cuSBF (insert_sequence_kmers_kernel, contains_sequence_kmers_kernel
// and their dense-packed twins).  Results are bit-identical to it; the work
// decomposition is new:
//
//   * A persistent CTA (two per SM) walks tiles of 8192 consecutive windows
//     (kTileKmers).  Each tile's input bytes are staged into shared memory by
//     a 1D bulk async copy (TMA) on an mbarrier, double-buffered and issued
//     two tiles ahead, so copies overlap hashing.  Only the 16-byte aligned
//     interior goes through the bulk copy; ragged edges are read with plain
//     loads, so nothing outside the caller's buffer is touched.  Every wait
//     is bounded and reports kDevErrStageTimeout instead of hanging.
//   * Staged bytes are encoded with SWAR into 2-bit code words (16 bases per
//     32-bit word, earliest base in the top bits) plus invalid masks.
//   * Each of the 256 threads owns a strip of 32 consecutive windows.  Every
//     m-mer and s-mer of the strip is a funnel shift of the code words,
//     every position is hashed once, and the per-window minimizer is a
//     Gil-Werman sliding minimum over blocks of W positions (about 3
//     comparisons per window for any W <= 16, where the reference hashes
//     and compares all W m-mers of every window).
//   * Insert merges consecutive windows that select the same shard (a
//     super-k-mer run) in registers and flushes each run with one 32-byte
//     bulk OR-reduction (cp.reduce.async.bulk .or.b64) from a per-thread
//     shared-memory ring: one L2 sector operation per run.
//   * Query copies each run head's 32-byte shard into per-thread shared
//     slots with cp.async as the heads are found, borrows the left
//     neighbour's staged shard when a run crosses the strip boundary, and
//     tests the findere rule (all k-s+1 s-mers present) per window.
//   * Insert word masks come from a shared one-hot table (1 << b).
//   * Ragged launches take tiles from a device work-queue counter and drop
//     windows that cross a record boundary or touch a byte outside every
//     record (marked per tile in shared memory).
#pragma once

#include "sbf_device.cuh"
#include "sbf_flush.cuh"
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
    static_assert(M >= 1 && M <= K, "m must satisfy 1 <= m <= k");
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
__device__ __forceinline__ void fill_ragged(const TileParams& p, const TileGeom& g, uint8_t* buf) {
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

// Expands the four low bits of `nib` into four 0/1 bytes (bit r -> byte r).
__device__ __forceinline__ uint32_t spread4(uint32_t nib) {
    return (nib * 0x00204081u) & 0x01010101u;
}

// ---------------------------------------------------------------------------
// Strip computation: kStrip consecutive windows per thread
// ---------------------------------------------------------------------------

// The 16 bases starting at strip position r, earliest base in bits 31:30.
// `c` holds the strip's code words; r is a compile-time constant after
// unrolling, so every access is a register.
__device__ __forceinline__ uint32_t win16(const uint32_t* c, int r) {
    const int q = r >> 4, s = r & 15;
    return s == 0 ? c[q] : __funnelshift_l(c[q + 1], c[q], 2 * s);
}

template <class C>
__device__ __forceinline__ uint64_t mh_at(const uint32_t* c, int r) {
    if constexpr (C::M > 16) {
        // Longer m-mers span two 16-base windows, like long s-mers.
        const uint64_t hi = win16(c, r) >> (2 * (32 - C::M));
        return mmer_hash((hi << 32) | win16(c, r + C::M - 16));
    } else {
        return mmer_hash(win16(c, r) >> (2 * (16 - C::M)));
    }
}

template <class C>
__device__ __forceinline__ uint64_t smer_at(const uint32_t* c, int r) {
    if constexpr (C::S > 16) {
        const uint64_t hi = win16(c, r) >> (2 * (32 - C::S));
        return (hi << 32) | win16(c, r + C::S - 16);
    } else {
        return win16(c, r) >> (2 * (16 - C::S));
    }
}

// Low word of min(a, b): the shard only needs the minimum's low 32 bits.
__device__ __forceinline__ uint32_t min64_lo(uint64_t a, uint64_t b) {
    return static_cast<uint32_t>(a < b ? a : b);
}

// Calls fn(j, shard) for the strip's windows j = 0..kStrip-1 in order.
// For 2 <= W <= 16 m-mers per window the minimum is a Gil-Werman sliding
// minimum over blocks of W positions: window b0 + r of the block starting at
// b0 is min(suffix_b0[r], prefix_{b0+W}[r-1]), about three 64-bit
// comparisons per window whatever W is (instead of W - 1).
template <class C, class Fn>
__device__ __forceinline__ void for_each_shard(const uint32_t* c, uint32_t shard_mask, Fn&& fn) {
    constexpr int W = C::W;
    if constexpr (W >= 2 && W <= 16) {
#pragma unroll
        for (int b0 = 0; b0 < kStrip; b0 += W) {
            uint64_t suf[W];
            suf[W - 1] = mh_at<C>(c, b0 + W - 1);
#pragma unroll
            for (int r = W - 2; r >= 0; --r) suf[r] = min64(mh_at<C>(c, b0 + r), suf[r + 1]);
            fn(b0, static_cast<uint32_t>(suf[0]) & shard_mask);
            uint64_t pre = ~uint64_t{0};
#pragma unroll
            for (int r = 1; r < W; ++r) {
                if (b0 + r < kStrip) {
                    pre = min64(pre, mh_at<C>(c, b0 + W - 1 + r));
                    fn(b0 + r, min64_lo(suf[r], pre) & shard_mask);
                }
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < kStrip; ++j) {
            uint64_t v = mh_at<C>(c, j);
#pragma unroll
            for (int o = 1; o < W; ++o) v = min64(v, mh_at<C>(c, j + o));
            fn(j, static_cast<uint32_t>(v) & shard_mask);
        }
    }
}

// Valid-window mask: window j holds K valid bases and lies in [0, n_kmers).
// inv[q] holds the invalid bits of code word q (bit r = base 16q + r).
template <class C>
__device__ __forceinline__ uint32_t strip_valid(const uint32_t* inv, int64_t first_kmer,
                                                uint64_t n_kmers) {
    uint32_t vmask = 0xFFFFFFFFu;
    const uint64_t bits = static_cast<uint64_t>(inv[0]) | (static_cast<uint64_t>(inv[1]) << 16) |
                          (static_cast<uint64_t>(inv[2]) << 32) |
                          (static_cast<uint64_t>(inv[3]) << 48);
    constexpr uint64_t kWin = (uint64_t{1} << C::K) - 1;
    if (bits) {
#pragma unroll
        for (int j = 0; j < kStrip; ++j)
            if ((bits >> j) & kWin) vmask &= ~(1u << j);
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

// One-hot word masks of the s-mer at strip position r.  With four hashes
// each word gets one bit, read from `onehot` (1 << b for b = 0..63 in the
// CTA's shared memory): four table loads replace four 64-bit variable
// shifts on the ALU pipe.
template <class C>
__device__ __forceinline__ void smer_masks(const uint32_t* c, int r, uint64_t m[4],
                                           const uint64_t* onehot) {
    const uint64_t h = smer_hash(smer_at<C>(c, r));
    if constexpr (C::H == 4) {
#pragma unroll
        for (int j = 0; j < 4; ++j) m[j] = onehot[bit_address<4>(h, j)];
    } else {
        m[0] = m[1] = m[2] = m[3] = 0;
#pragma unroll
        for (int j = 0; j < C::H; ++j) m[j & 3] |= uint64_t{1} << bit_address<C::H>(h, j);
    }
}

// Fills the one-hot table of smer_masks (threads 0..63; the caller's next
// barrier publishes it).
__device__ __forceinline__ void onehot_init(uint64_t* onehot) {
    if (threadIdx.x < 64) onehot[threadIdx.x] = uint64_t{1} << threadIdx.x;
}

// Insert: the mask of window j is T_j = OR of the one-hot masks of its F
// s-mers; a super-k-mer run (consecutive valid windows with equal shard)
// accumulates acc = OR T_j and is handed to flush(end, shard, acc) with end
// non-zero when the next window leaves the run (the insert kernel ORs it
// into the shard; the sharded insert's emit kernel records it).  With four
// s-mers per window, flush is called on every window with `end` as its
// predicate, so the per-run work needs no branch.
template <class C, class Flush>
__device__ __forceinline__ void insert_strip(const uint32_t* c, uint32_t vmask,
                                             uint32_t shard_mask, const uint64_t* onehot,
                                             Flush&& flush) {
    constexpr int F = C::F;
    uint64_t acc[4] = {0, 0, 0, 0};
    uint32_t prev_shard = 0;
    bool prev_valid = false;
    if constexpr (F == 4) {
        // T_j = P_j | P_{j+2} with pair masks P_x = m_x | m_{x+1}.
        uint64_t m0[4], m1[4], m2[4];
        smer_masks<C>(c, 0, m0, onehot);
        smer_masks<C>(c, 1, m1, onehot);
        smer_masks<C>(c, 2, m2, onehot);
        uint64_t pa[4], pb[4];
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            pa[w] = m0[w] | m1[w];
            pb[w] = m1[w] | m2[w];
        }
        for_each_shard<C>(c, shard_mask, [&](int j, uint32_t shard) {
            uint64_t m3[4];
            smer_masks<C>(c, j + 3, m3, onehot);
            const bool valid = (vmask >> j) & 1u;
            const bool cont = valid && prev_valid && shard == prev_shard;
            flush((prev_valid && !cont) ? 1u : 0u, prev_shard, acc);
            const uint64_t keep = cont ? ~uint64_t{0} : uint64_t{0};
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                const uint64_t pc = m2[w] | m3[w];
                acc[w] = (acc[w] & keep) | pa[w] | pc;
                pa[w] = pb[w];
                pb[w] = pc;
                m2[w] = m3[w];
            }
            prev_shard = shard;
            prev_valid = valid;
        });
    } else {
        uint64_t mring[F][4];
#pragma unroll
        for (int o = 0; o < F - 1; ++o) smer_masks<C>(c, o, mring[o], onehot);
        for_each_shard<C>(c, shard_mask, [&](int j, uint32_t shard) {
            smer_masks<C>(c, j + F - 1, mring[(j + F - 1) % F], onehot);
            const bool valid = (vmask >> j) & 1u;
            const bool cont = valid && prev_valid && shard == prev_shard;
            if (prev_valid && !cont) flush(1u, prev_shard, acc);
            const uint64_t keep = cont ? ~uint64_t{0} : uint64_t{0};
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                uint64_t t = mring[j % F][w];
#pragma unroll
                for (int o = 1; o < F; ++o) t |= mring[(j + o) % F][w];
                acc[w] = (acc[w] & keep) | t;
            }
            prev_shard = shard;
            prev_valid = valid;
        });
    }
    if (prev_valid) flush(1u, prev_shard, acc);
}

// Query shard slots: the run heads of a strip fetch their 32-byte shards into
// per-thread shared-memory slots with cp.async, all at once, so a thread has
// every shard load of its strip in flight while it hashes the strip's s-mers.
static_assert(kSlots * kThreads * 32 + kOverflow * kThreads * 4 == kQuerySlotBytes,
              "slot geometry");

// Half of a shard into a slot.  The .L2::64B fetch size makes an L2 miss
// fill 64 bytes instead of 128: a random 32-byte shard then costs about 64 B
// of DRAM reads instead of about 120 (measured with random sector reads on
// the B200), at the same speed.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.cg.shared.global.L2::64B [%0], [%1], 16;" ::"r"(smem_addr(smem_dst)),
                 "l"(gmem_src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ void load_shard_now(const uint64_t* p, uint64_t w[4]) {
    asm volatile("ld.global.nc.L2::64B.v4.u64 {%0, %1, %2, %3}, [%4];"
                 : "=l"(w[0]), "=l"(w[1]), "=l"(w[2]), "=l"(w[3])
                 : "l"(p));
}

// The H = 4 bit addresses of the s-mer at strip position r, one per byte:
// byte j is the bit of shard word j.
template <class C>
__device__ __forceinline__ uint32_t smer_bytes4(const uint32_t* c, int r) {
    const uint64_t h = smer_hash(smer_at<C>(c, r));
    const uint32_t lo = static_cast<uint32_t>(h), hi = static_cast<uint32_t>(h >> 32);
    // lo bits 0-5 -> word 0, lo bits 16-21 -> word 1, hi bits 0-5 -> word 2,
    // hi bits 16-21 -> word 3.
    const uint32_t a = lo & 0x003F003Fu;           // b0 in byte 0, b1 in byte 2
    const uint32_t b = (hi & 0x003F003Fu) << 8;    // b2 in byte 1, b3 in byte 3
    return __byte_perm(a | b, 0u, 0x3120u);        // bytes b0 b1 b2 b3
}

// The same four bit addresses, one per word: b[j] is the bit of shard word j.
template <class C>
__device__ __forceinline__ void smer_addr4(const uint32_t* c, int r, uint32_t b[4]) {
    const uint64_t h = smer_hash(smer_at<C>(c, r));
    const uint32_t lo = static_cast<uint32_t>(h), hi = static_cast<uint32_t>(h >> 32);
    b[0] = lo & 63u;
    b[1] = (lo >> 16) & 63u;
    b[2] = hi & 63u;
    b[3] = (hi >> 16) & 63u;
}

template <class C>
__device__ __forceinline__ uint32_t smer_present_h(uint64_t h, const uint64_t* w) {
    uint32_t acc = 0xFFFFFFFFu;
#pragma unroll
    for (int j = 0; j < C::H; ++j) acc &= static_cast<uint32_t>(w[j & 3] >> bit_address<C::H>(h, j));
    return acc;
}

__device__ __forceinline__ void store_strip_bytes(uint32_t result, uint8_t* out, int64_t first_kmer,
                                                  uint64_t n_kmers) {
    if (first_kmer >= 0 && first_kmer + kStrip <= static_cast<int64_t>(n_kmers)) {
        uint4 v0, v1;
        v0.x = spread4(result & 0xFu);
        v0.y = spread4((result >> 4) & 0xFu);
        v0.z = spread4((result >> 8) & 0xFu);
        v0.w = spread4((result >> 12) & 0xFu);
        v1.x = spread4((result >> 16) & 0xFu);
        v1.y = spread4((result >> 20) & 0xFu);
        v1.z = spread4((result >> 24) & 0xFu);
        v1.w = spread4(result >> 28);
        uint4* dst = reinterpret_cast<uint4*>(out + first_kmer);
        dst[0] = v0;
        dst[1] = v1;
    } else {
#pragma unroll
        for (int j = 0; j < kStrip; ++j) {
            const int64_t i = first_kmer + j;
            if (i >= 0 && i < static_cast<int64_t>(n_kmers))
                out[i] = static_cast<uint8_t>((result >> j) & 1u);
        }
    }
}

// Loads shard slot words x[0..7] from shared address `addr` when `pred` is
// non-zero and leaves them unchanged otherwise: a predicated load, so a run
// head costs no branch in the per-window loop.
__device__ __forceinline__ void lds_slot_if(uint32_t pred, uint32_t addr, uint32_t (&x)[8]) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %8, 0;\n\t"
        "@p ld.shared.v4.u32 {%0, %1, %2, %3}, [%9];\n\t"
        "@p ld.shared.v4.u32 {%4, %5, %6, %7}, [%9+16];\n\t}"
        : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4]), "+r"(x[5]), "+r"(x[6]),
          "+r"(x[7])
        : "r"(pred), "r"(addr));
}

// Query of one strip without slots: each run head loads its shard when it is
// reached.  Used for strips with more run heads than slots.
template <class C>
__device__ __noinline__ uint32_t query_strip_direct(const uint32_t* c, uint32_t vmask,
                                                    uint32_t shard_mask, const uint64_t* words) {
    constexpr int F = C::F;
    uint64_t ring[F];
#pragma unroll
    for (int o = 0; o < F - 1; ++o) ring[o] = smer_hash(smer_at<C>(c, o));
    uint64_t w[4] = {0, 0, 0, 0};
    bool have = false;
    uint32_t cur = 0, result = 0;
    for_each_shard<C>(c, shard_mask, [&](int j, uint32_t sh) {
        ring[(j + F - 1) % F] = smer_hash(smer_at<C>(c, j + F - 1));
        const bool valid = (vmask >> j) & 1u;
        if (valid && (!have || sh != cur)) {
            load_shard_now(words + static_cast<uint64_t>(sh) * 4, w);
            cur = sh;
            have = true;
        }
        uint32_t present = valid ? 1u : 0u;
#pragma unroll
        for (int o = 0; o < F; ++o) present &= smer_present_h<C>(ring[(j + o) % F], w);
        result |= (present & 1u) << j;
    });
    return result;
}

// Query of one strip: minimizers -> cp.async of every run head's shard into
// the thread's slots (issued as the heads are found) -> s-mer hashing while
// the copies are in flight -> wait -> findere tests -> output bytes.
// kAddrInLoop (four hashes): compute each position's bit addresses as it
// enters the window instead of packing the strip's addresses while the
// copies fly.  It frees 35 registers and makes the plain <31,28,16,4> query
// 1.1% faster, but spills in the ragged kernels and with one s-mer per
// window, which keep the packed form.
template <class C, bool kAddrInLoop>
__device__ __forceinline__ uint32_t query_strip(const uint32_t* c, uint32_t vmask, uint32_t shard_mask,
                                            const uint64_t* words, uint64_t* slot0,
                                            uint32_t* ovf0, uint8_t* out, int64_t first_kmer,
                                            uint64_t n_kmers) {
    // Slot n of this thread lives at slot0 + n * kThreads * 4 and overflow
    // entry e at ovf0 + e * kThreads ([entry][thread] layouts: neighbouring
    // threads touch neighbouring addresses).
    constexpr int kSlotStride = kThreads * 4;
    constexpr int F = C::F;
    // Run heads: a valid window whose predecessor is invalid or selects
    // another shard.  The first kSlots heads copy their shard into slots; the
    // next kOverflow only record their shard id (loaded when reached).  The
    // copy for window 0 is decided after the loop: when the left neighbour's
    // last run continues into this strip (same shard, both ends valid), its
    // staged slot is read instead of loading the sector again.
    uint32_t heads = 0;
    int n = 0;
    uint32_t first_sh = 0, last_sh = 0;
    {
        uint32_t prev = 0;
        for_each_shard<C>(c, shard_mask, [&](int j, uint32_t sh) {
            const bool valid = (vmask >> j) & 1u;
            const bool prev_valid = j > 0 && ((vmask >> (j - 1)) & 1u);
            if (j == 0) first_sh = sh;
            if (j == kStrip - 1) last_sh = sh;
            if (valid && (!prev_valid || sh != prev)) {
                heads |= 1u << j;
                if (j > 0) {
                    if (n < kSlots) {
                        const uint64_t* src = words + static_cast<uint64_t>(sh) * 4;
                        uint64_t* dst = slot0 + n * kSlotStride;
                        cp_async16(dst, src);
                        cp_async16(dst + 2, src + 2);
                    } else if (n < kSlots + kOverflow) {
                        ovf0[(n - kSlots) * kThreads] = sh;
                    }
                }
                ++n;
            }
            prev = sh;
        });
    }
    const int lane = threadIdx.x & 31;
    const bool last_open = (vmask >> (kStrip - 1)) & 1u;
    // Lend the last run's slot only when its head is not window 0: window 0's
    // slot may itself be borrowed (never loaded), so lending it would chain.
    const bool last_is_w0 = n == 1 && (vmask & 1u);
    const int my_last_slot = last_open && n >= 1 && n <= kSlots && !last_is_w0 ? n - 1 : -1;
    const uint32_t left_sh = __shfl_up_sync(0xFFFFFFFFu, last_sh, 1);
    const int left_slot = __shfl_up_sync(0xFFFFFFFFu, my_last_slot, 1);
    const bool borrow = lane > 0 && (vmask & 1u) && left_slot >= 0 && left_sh == first_sh;
    if ((vmask & 1u) && !borrow) {
        const uint64_t* src = words + static_cast<uint64_t>(first_sh) * 4;
        cp_async16(slot0, src);
        cp_async16(slot0 + 2, src + 2);
    }
    cp_async_commit();
    if (n > kSlots + kOverflow) {
        cp_async_wait_all();
        __syncwarp();
        const uint32_t direct = query_strip_direct<C>(c, vmask, shard_mask, words);
        if (out) store_strip_bytes(direct, out, first_kmer, n_kmers);
        return direct;
    }
    // Hash the strip's s-mers while the shard copies are in flight (with
    // four hashes, one word of bit addresses per position), unless
    // kAddrInLoop computes them as the positions enter the window.
    constexpr int NP = kStrip + F - 1;
    constexpr bool kPacked = C::H == 4 && !kAddrInLoop;
    uint32_t bytes[kPacked ? NP : 1];
    uint64_t hs[C::H == 4 ? 1 : NP];
#pragma unroll
    for (int r = 0; r < NP; ++r) {
        if constexpr (kPacked)
            bytes[r] = smer_bytes4<C>(c, r);
        else if constexpr (C::H != 4)
            hs[r] = smer_hash(smer_at<C>(c, r));
    }
    cp_async_wait_all();
    __syncwarp();  // neighbours' slots are complete before any is borrowed
    uint64_t w[4] = {0, 0, 0, 0};
    uint32_t result = 0;
    // Bit addresses of the F positions of the current window, extracted once
    // per position as it enters the window.
    uint32_t ring[C::H == 4 ? F : 1][4];
    auto enter = [&](int r) {  // position r enters the window
        if constexpr (kPacked) {
#pragma unroll
            for (int q = 0; q < 4; ++q) ring[r % F][q] = __byte_perm(bytes[r], 0u, 0x4440u + q);
        } else if constexpr (C::H == 4) {
            smer_addr4<C>(c, r, ring[r % F]);
        }
    };
#pragma unroll
    for (int o = 0; o < F - 1; ++o) enter(o);
    // (Configurations with one s-mer per window or sixteen hashes keep the
    // branching loop below: the predicated form spills registers there.)
    constexpr bool kPredicated = F > 1 && C::H <= 8;
    if (kPredicated && n <= kSlots) {
        // Every head's shard is in a slot (the common case): each window
        // does a predicated load of the next head's slot and advances the
        // slot address when it is a head, so the loop has no per-head branch.
        const uint64_t* sfirst = borrow ? slot0 + left_slot * kSlotStride - 4 : slot0;
        uint32_t addr = smem_addr(sfirst);
        const uint32_t base = smem_addr(slot0);
        uint32_t x[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        uint32_t loaded = 0;
#pragma unroll
        for (int j = 0; j < kStrip; ++j) {
            enter(j + F - 1);
            const uint32_t head = (heads >> j) & 1u;
            lds_slot_if(head, addr, x);
            loaded += head;
            addr = head ? base + loaded * (kSlotStride * 8) : addr;
#pragma unroll
            for (int q = 0; q < 4; ++q) w[q] = (static_cast<uint64_t>(x[2 * q + 1]) << 32) | x[2 * q];
            uint32_t present = (vmask >> j) & 1u;
#pragma unroll
            for (int o = 0; o < F; ++o) {
                if constexpr (C::H == 4) {
                    const uint32_t* b = ring[(j + o) % F];
                    present &= static_cast<uint32_t>(w[0] >> b[0]) & static_cast<uint32_t>(w[1] >> b[1]) &
                               static_cast<uint32_t>(w[2] >> b[2]) & static_cast<uint32_t>(w[3] >> b[3]);
                } else {
                    present &= smer_present_h<C>(hs[j + o], w);
                }
            }
            result |= (present & 1u) << j;
        }
        if (out) store_strip_bytes(result, out, first_kmer, n_kmers);
        return result;
    }
    // More heads than slots: the later heads load their shards directly.
    n = 0;
#pragma unroll
    for (int j = 0; j < kStrip; ++j) {
        enter(j + F - 1);
        if ((heads >> j) & 1u) {
            if (n < kSlots) {
                // Slot 0 may be the left neighbour's last slot (its thread's
                // slots sit 4 words below this thread's).
                const uint64_t* sn = (n == 0 && borrow) ? slot0 + left_slot * kSlotStride - 4
                                                        : slot0 + n * kSlotStride;
                const uint4 lo = *reinterpret_cast<const uint4*>(sn);
                const uint4 hi = *reinterpret_cast<const uint4*>(sn + 2);
                w[0] = (static_cast<uint64_t>(lo.y) << 32) | lo.x;
                w[1] = (static_cast<uint64_t>(lo.w) << 32) | lo.z;
                w[2] = (static_cast<uint64_t>(hi.y) << 32) | hi.x;
                w[3] = (static_cast<uint64_t>(hi.w) << 32) | hi.z;
            } else {
                load_shard_now(words + static_cast<uint64_t>(ovf0[(n - kSlots) * kThreads]) * 4, w);
            }
            ++n;
        }
        uint32_t present = (vmask >> j) & 1u;
#pragma unroll
        for (int o = 0; o < F; ++o) {
            if constexpr (C::H == 4) {
                const uint32_t* b = ring[(j + o) % F];
                present &= static_cast<uint32_t>(w[0] >> b[0]) & static_cast<uint32_t>(w[1] >> b[1]) &
                           static_cast<uint32_t>(w[2] >> b[2]) & static_cast<uint32_t>(w[3] >> b[3]);
            } else {
                present &= smer_present_h<C>(hs[j + o], w);
            }
        }
        result |= (present & 1u) << j;
    }
    if (out) store_strip_bytes(result, out, first_kmer, n_kmers);
    return result;
}

// ---------------------------------------------------------------------------
// The tile kernel
// ---------------------------------------------------------------------------

// Ragged launches: marks the record structure of the staged tile.  brk bit
// r of word q is set when tile position 16q + r starts a record (windows
// that contain it and the byte before it span two records); bytes outside
// every record are added to the invalid bits.  Each thread takes records
// first, first + kThreads, ... of those overlapping the tile.
template <class C>
__device__ __forceinline__ void mark_records(const TileParams& p, int64_t s0, uint32_t first,
                                             uint32_t* inval, uint32_t* brk) {
    constexpr int64_t kSpan = kCodeWords * 16;
    const int64_t len = static_cast<int64_t>(p.input_bytes);
    const int64_t t_end = s0 + kSpan;
    auto set_bits = [&](uint32_t* arr, int64_t a, int64_t b) {  // dense [a, b)
        a = a > s0 ? a : s0;
        b = b < t_end ? b : t_end;
        for (int64_t x = a; x < b;) {
            const int64_t pos = x - s0;
            const int q = static_cast<int>(pos >> 4), r = static_cast<int>(pos & 15);
            const int64_t n = (16 - r) < (b - x) ? (16 - r) : (b - x);
            atomicOr(arr + q, ((1u << n) - 1u) << r);
            x += n;
        }
    };
    const uint64_t n = p.n_ranges;
    if (threadIdx.x == 0) {
        // Bytes before the first overlapping record.
        const int64_t gap0 = first == 0 ? 0
                                        : static_cast<int64_t>(p.ranges[first - 1].offset +
                                                               p.ranges[first - 1].bytes);
        const int64_t until = first < n ? static_cast<int64_t>(p.ranges[first].offset) : len;
        set_bits(inval, gap0, until);
    }
    for (uint64_t r = first + threadIdx.x; r < n; r += kThreads) {
        const DevRange rec = p.ranges[r];
        const int64_t a = static_cast<int64_t>(rec.offset);
        if (a >= t_end) break;
        const int64_t b = a + static_cast<int64_t>(rec.bytes);
        if (a > s0 && a < t_end) {
            const int64_t pos = a - s0;
            atomicOr(brk + (pos >> 4), 1u << (pos & 15));
        }
        const int64_t next = r + 1 < n ? static_cast<int64_t>(p.ranges[r + 1].offset) : len;
        if (next > b) set_bits(inval, b, next);
    }
}

// Ragged launches: clears windows j of the strip that contain a record start
// other than their own first byte.
template <class C>
__device__ __forceinline__ uint32_t strip_in_record(const uint32_t* bk, uint32_t vmask) {
    const uint64_t bits = static_cast<uint64_t>(bk[0]) | (static_cast<uint64_t>(bk[1]) << 16) |
                          (static_cast<uint64_t>(bk[2]) << 32) |
                          (static_cast<uint64_t>(bk[3]) << 48);
    constexpr uint64_t kInner = ((uint64_t{1} << C::K) - 1) >> 1;  // positions j+1 .. j+K-1
    if (bits) {
#pragma unroll
        for (int j = 0; j < kStrip; ++j)
            if ((bits >> (j + 1)) & kInner) vmask &= ~(1u << j);
    }
    return vmask;
}

// Ragged launches with per-record tallies: adds the strip's valid windows
// (vmask) and positive windows (hits) to the records they belong to.  Window
// j belongs to the record containing byte x0 + j.  The strip's records are
// found by one binary search (first record ending after its first valid
// window) and a walk over the record ends; empty records are skipped by the
// walk.  Across the warp, the record a strip starts in is usually the one the
// previous strip ended in: a strip's last record is handed to the next lane
// when it is that lane's first, and lanes holding the same record are summed
// with one match + reduce, so a warp issues about one atomic pair per record
// it touches (count_positive_kmers_per_record_kernel,
// detail/count_positive_kmers.cuh:21-45, fused into the query epilogue).
__device__ __forceinline__ void tally_records(const TileParams& p, uint32_t first, int64_t x0,
                                              uint32_t vmask, uint32_t hits) {
    constexpr uint32_t kNone = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t n = p.n_ranges;
    uint32_t kf = kNone, vf = 0, kl = kNone, vl = 0;  // first / last record and (valid << 16 | pos)
    auto add = [&](uint32_t r, uint32_t c) {
        const uint64_t at = static_cast<uint64_t>(r) << p.rec_shift;
        atomicAdd(p.rec_valid + at, static_cast<unsigned long long>(c >> 16));
        if (c & 0xFFFFu) atomicAdd(p.rec_pos + at, static_cast<unsigned long long>(c & 0xFFFFu));
    };
    uint32_t v = vmask;
    const uint32_t h = hits & vmask;
    if (v) {
        int j = __ffs(v) - 1;
        // First record whose end exceeds x0 + j (records before `first` end
        // before the tile).
        uint64_t lo = first, hi = n;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (static_cast<int64_t>(p.ranges[mid].offset + p.ranges[mid].bytes) > x0 + j)
                hi = mid;
            else
                lo = mid + 1;
        }
        uint64_t r = lo;
        for (bool head = true; r < n; head = false) {
            const int64_t lim = static_cast<int64_t>(p.ranges[r].offset + p.ranges[r].bytes) - x0;
            const uint32_t seg = lim >= 32 ? v : (v & ((1u << lim) - 1u));
            const uint32_t c = (static_cast<uint32_t>(__popc(seg)) << 16) |
                               static_cast<uint32_t>(__popc(h & seg));
            v &= ~seg;
            if (head) {
                kf = static_cast<uint32_t>(r);
                vf = c;
            } else if (v) {
                add(static_cast<uint32_t>(r), c);  // a record inside the strip
            } else {
                kl = static_cast<uint32_t>(r);
                vl = c;
            }
            if (!v) break;
            j = __ffs(v) - 1;
            do {
                ++r;
            } while (r < n && static_cast<int64_t>(p.ranges[r].offset + p.ranges[r].bytes) <= x0 + j);
        }
    }
    const uint32_t prev_kl = __shfl_up_sync(0xFFFFFFFFu, kl, 1);
    const uint32_t prev_vl = __shfl_up_sync(0xFFFFFFFFu, vl, 1);
    const uint32_t next_kf = __shfl_down_sync(0xFFFFFFFFu, kf, 1);
    if (lane > 0 && prev_kl != kNone && prev_kl == kf) vf += prev_vl;
    if (kl != kNone && !(lane < 31 && next_kf == kl)) add(kl, vl);
    const uint32_t grp = __match_any_sync(0xFFFFFFFFu, kf);
    const uint32_t tot = __reduce_add_sync(grp, vf);
    if (kf != kNone && lane == static_cast<uint32_t>(__ffs(grp) - 1)) add(kf, tot);
}

// Persistent tile kernel.  Plain launches walk tiles blockIdx.x + i * gridDim.x;
// ragged launches take tiles from the device work-queue counter p.queue, so
// tiles of uneven cost (records of any length, N runs) balance across CTAs.
// Either way tile i+2 is known while tile i is processed, so its staging copy
// is issued two tiles ahead.
template <class C, bool kQuery, bool kDense, bool kRagged>
__global__ void __launch_bounds__(kThreads, 2) tile_kernel(TileParams p) {
    __shared__ alignas(128) uint8_t stage[2][kStageBytes];
    __shared__ uint32_t code[kCodeWords + 4];
    __shared__ uint32_t inval[kCodeWords + 4];
    __shared__ uint32_t brk[kRagged ? kCodeWords + 4 : 1];
    __shared__ uint64_t tiles[3];
    __shared__ uint32_t first_rec[3];
    __shared__ unsigned long long tally[2];
    __shared__ alignas(8) uint64_t bars[2];
    __shared__ uint64_t onehot[kQuery ? 1 : 64];

    const int tid = threadIdx.x;
    if constexpr (!kQuery) onehot_init(onehot);
    if constexpr (kRagged) {
        if (p.sizes) {
            const DevSizes z = *p.sizes;
            p.input_bytes = z.input_bytes;
            p.n_kmers = z.n_kmers;
            p.n_tiles = z.n_tiles;
            p.n_ranges = z.n_ranges;
        }
    }
    auto take = [&](uint32_t i, int slot) {
        uint64_t t;
        if constexpr (kRagged) {
            t = atomicAdd(p.queue, 1u);
            first_rec[slot] = t < p.n_tiles ? p.tile_rec[t] : 0u;
        } else {
            t = blockIdx.x + static_cast<uint64_t>(i) * gridDim.x;
        }
        tiles[slot] = t;
        return t;
    };
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
        tally[0] = tally[1] = 0;
        const uint64_t t0 = take(0, 0), t1 = take(1, 1);
        if (t0 < p.n_tiles) issue_stage<kDense>(p, t0, stage[0], &bars[0]);
        if (t1 < p.n_tiles) issue_stage<kDense>(p, t1, stage[1], &bars[1]);
    }
    __syncthreads();
    // Dynamic shared memory, [slot][thread] layout: the query kernel's shard
    // slots (kQuerySlotBytes per CTA) or the insert kernel's flush staging
    // ring (kInsertSlotBytes per CTA).
    extern __shared__ __align__(16) uint64_t slots[];
    FlushRing ring{slots + 4 * tid, 0u};
    (void)ring;
    unsigned long long n_valid = 0, n_pos = 0;
    for (uint32_t it = 0;; ++it) {
        const uint64_t tile = tiles[it % 3];
        if (tile >= p.n_tiles) break;
        const int b = it & 1;
        const uint32_t parity = (it >> 1) & 1u;
        const bool ok = mbar_wait_bounded(&bars[b], parity);
        if (__syncthreads_or(!ok)) {
            // Both staging buffers may still have a bulk copy in flight:
            // this tile's (whose wait ran out) and the next tile's.  Give
            // each one more bounded wait before the CTA's shared memory is
            // released, so no copy lands in memory a later CTA owns.
            if (tid == 0) {
                atomicExch(p.err, kDevErrStageTimeout);
                (void)mbar_wait_bounded(&bars[b], parity);
                if (tiles[(it + 1) % 3] < p.n_tiles)
                    (void)mbar_wait_bounded(&bars[b ^ 1], ((it + 1) >> 1) & 1u);
            }
            __syncthreads();
            if constexpr (!kQuery) flush_ring_drain();
            return;
        }
        const TileGeom g = tile_geom<kDense>(p, tile);
        fill_ragged<kDense>(p, g, stage[b]);
        __syncthreads();
        for (int q = tid; q < kCodeWords; q += kThreads) {
            uint32_t cw, iv;
            encode_word<kDense>(g, stage[b], q, cw, iv);
            code[q] = cw;
            inval[q] = iv;
            if constexpr (kRagged) brk[q] = 0u;
        }
        if constexpr (kRagged) {
            __syncthreads();
            mark_records<C>(p, g.s0, first_rec[it % 3], inval, brk);
        }
        __syncthreads();
        if (tid == 0) {
            const uint64_t t2 = take(it + 2, (it + 2) % 3);
            if (t2 < p.n_tiles) issue_stage<kDense>(p, t2, stage[b], &bars[b]);
        }

        uint32_t c[kStripWords], iv[kStripWords];
#pragma unroll
        for (int q = 0; q < kStripWords; ++q) {
            c[q] = code[tid * (kStrip / 16) + q];
            iv[q] = inval[tid * (kStrip / 16) + q];
        }
        const int64_t first_kmer = g.s0 + static_cast<int64_t>(tid) * kStrip;
        uint32_t vmask = strip_valid<C>(iv, first_kmer, p.n_kmers);
        if constexpr (kRagged) {
            uint32_t bk[kStripWords];
#pragma unroll
            for (int q = 0; q < kStripWords; ++q) bk[q] = brk[tid * (kStrip / 16) + q];
            vmask = strip_in_record<C>(bk, vmask);
            n_valid += __popc(vmask);
        }
        uint32_t hits = 0;
        if constexpr (kQuery) {
            constexpr bool kAddrInLoop = !kRagged && C::W == 16 && C::F > 1;
            hits = query_strip<C, kAddrInLoop>(
                c, vmask, p.shard_mask, p.words, slots + 4 * tid,
                reinterpret_cast<uint32_t*>(slots + kSlots * kThreads * 4) + tid, p.out,
                first_kmer, p.n_kmers);
            if constexpr (kRagged) n_pos += __popc(hits & vmask);
            // Bit-packed mode (grid phase 0, so strips start at multiples of
            // 32 windows): one 32-bit word per strip, coalesced across the warp.
            if (p.out_bits && first_kmer < static_cast<int64_t>(p.n_kmers))
                p.out_bits[first_kmer >> 5] = hits;
        } else {
            if (vmask)
                insert_strip<C>(c, vmask, p.shard_mask, onehot,
                                [&](uint32_t end, uint32_t shard, const uint64_t* acc) {
                                    flush_run_if(end, p.words, shard, acc, ring);
                                });
        }
        if constexpr (kRagged) {
            if (p.rec_valid) tally_records(p, first_rec[it % 3], first_kmer, vmask, hits);
        }
    }
    if constexpr (!kQuery) flush_ring_drain();
    if constexpr (kRagged) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            n_valid += __shfl_down_sync(0xFFFFFFFFu, n_valid, o);
            n_pos += __shfl_down_sync(0xFFFFFFFFu, n_pos, o);
        }
        if ((tid & 31) == 0) {
            atomicAdd(&tally[0], n_valid);
            atomicAdd(&tally[1], n_pos);
        }
        __syncthreads();
        if (tid == 0) {
            atomicAdd(p.counts, tally[0]);
            atomicAdd(p.counts + 1, tally[1]);
        }
    }
}

}  // namespace sbf
