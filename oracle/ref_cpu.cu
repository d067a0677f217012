// ref_cpu.cu -- host-side driver over the reference cuSBF's own arithmetic.
//
// TEST INFRASTRUCTURE ONLY (built into oracle/_ref/, never shipped).  It is
// compiled by oracle/Makefile directly against the reference headers
// (include/cusbf/*.cuh of tdortman/cuSBF) and calls the reference's
// host-callable primitives:
//   Config<...>::Alphabet::encode            include/cusbf/Alphabet.cuh:132-141
//   detail::extractPackedSubwindow           include/cusbf/detail/filter_common.cuh:129-134
//   detail::minimizer_hash64, detail::hash64 include/cusbf/hashutil.cuh:192-209
//   filter_block<Config>::sectorizedBitAddress include/cusbf/detail/filter_impl.cuh:37-48
//   filter_ref<Config>::shard_index          include/cusbf/filter_ref.cuh:52-55
// The loops around them follow include/cusbf/detail/kernels.cuh:107-172
// (insert) and :40-99 (query) one window at a time, so the result is the
// reference's word array and hit bytes computed by the reference's code on
// the CPU.  It pins oracle/sbf_oracle.c and generates tests/golden/.
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include <cusbf/Alphabet.cuh>
#include <cusbf/config.cuh>
#include <cusbf/detail/filter_common.cuh>
#include <cusbf/detail/filter_impl.cuh>
#include <cusbf/hashutil.cuh>

namespace {

template <typename C>
struct RefOps {
    using Block = cusbf::filter_block<C>;

    static bool window(const uint8_t* sym, uint64_t i, uint64_t num_shards, bool dense,
                       uint32_t& shard, uint64_t masks[4]) {
        uint64_t packed = 0;
        for (uint64_t j = 0; j < C::k; ++j) {
            const uint8_t e = sym[i + j];
            if (!dense && e == C::Alphabet::invalidSymbol) return false;
            packed = (packed << C::symbolBits) | (e & C::symbolMask);
        }
        uint64_t minh = cusbf::detail::kInvalidHash;
        for (uint64_t o = 0; o < C::minimizerSpan; ++o) {
            const uint64_t mm = cusbf::detail::extractPackedSubwindow<C, C::m, C::k>(packed, o);
            const uint64_t hh = cusbf::detail::minimizer_hash64(mm);
            minh = hh < minh ? hh : minh;
        }
        shard = static_cast<uint32_t>(minh & (num_shards - 1));
        masks[0] = masks[1] = masks[2] = masks[3] = 0;
        for (uint64_t o = 0; o < C::findereSpan; ++o) {
            const uint64_t sm = cusbf::detail::extractPackedSubwindow<C, C::s, C::k>(packed, o);
            const uint64_t hs = cusbf::detail::hash64(sm);
            cusbf::detail::forEachHashIndex<C>(
                [&]<uint64_t J>(std::integral_constant<uint64_t, J>) {
                    masks[J % C::blockWordCount] |= uint64_t{1}
                                                    << Block::template sectorizedBitAddress<J>(hs);
                });
        }
        return true;
    }

    static std::vector<uint8_t> encode(const char* seq, uint64_t len) {
        const uint64_t n = len / C::symbolWidth;
        std::vector<uint8_t> sym(n);
        for (uint64_t t = 0; t < n; ++t) sym[t] = C::Alphabet::encode(seq + t * C::symbolWidth);
        return sym;
    }

    static std::vector<uint8_t> decode_dense(const uint64_t* words, uint64_t n) {
        constexpr uint64_t per = 64 / C::symbolBits;
        std::vector<uint8_t> sym(n);
        for (uint64_t t = 0; t < n; ++t)
            sym[t] = static_cast<uint8_t>((words[t / per] >> ((t % per) * C::symbolBits)) &
                                          C::symbolMask);
        return sym;
    }

    template <typename Fn>
    static void parallel(uint64_t n, int threads, Fn fn) {
        if (threads < 1) threads = 1;
        if (static_cast<uint64_t>(threads) > n) threads = n ? static_cast<int>(n) : 1;
        const uint64_t per = (n + threads - 1) / threads;
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t) {
            const uint64_t b = std::min<uint64_t>(n, t * per);
            const uint64_t e = std::min<uint64_t>(n, b + per);
            pool.emplace_back([=] { fn(b, e); });
        }
        for (auto& th : pool) th.join();
    }

    static void insert_syms(const std::vector<uint8_t>& sym, bool dense, uint64_t* words,
                            uint64_t num_shards, int threads) {
        const uint64_t n = sym.size() < C::k ? 0 : sym.size() - C::k + 1;
        parallel(n, threads, [&](uint64_t b, uint64_t e) {
            uint64_t masks[4];
            uint32_t shard;
            for (uint64_t i = b; i < e; ++i) {
                if (!window(sym.data(), i, num_shards, dense, shard, masks)) continue;
                for (int q = 0; q < 4; ++q)
                    if (masks[q])
                        __atomic_fetch_or(&words[uint64_t{shard} * 4 + q], masks[q],
                                          __ATOMIC_RELAXED);
            }
        });
    }

    static void contains_syms(const std::vector<uint8_t>& sym, bool dense, const uint64_t* words,
                              uint64_t num_shards, uint8_t* out, int threads) {
        const uint64_t n = sym.size() < C::k ? 0 : sym.size() - C::k + 1;
        parallel(n, threads, [&](uint64_t b, uint64_t e) {
            uint64_t masks[4];
            uint32_t shard;
            for (uint64_t i = b; i < e; ++i) {
                if (!window(sym.data(), i, num_shards, dense, shard, masks)) {
                    out[i] = 0;
                    continue;
                }
                const uint64_t* w = words + uint64_t{shard} * 4;
                bool present = true;
                for (int q = 0; q < 4; ++q) present &= (w[q] & masks[q]) == masks[q];
                out[i] = present;
            }
        });
    }
};

using C31 = cusbf::Config<31, 28, 16, 4>;
using C31h8 = cusbf::Config<31, 28, 16, 8>;
using C31h16 = cusbf::Config<31, 28, 16, 16>;
using C5 = cusbf::Config<5, 4, 3, 4>;
using C21 = cusbf::Config<21, 19, 11, 4>;
using CProt = cusbf::Config<5, 4, 3, 4, 256, cusbf::ProteinAlphabet>;
using CTrip = cusbf::Config<3, 2, 2, 4, 256, cusbf::DnaTripletAlphabet>;

template <typename Fn>
int dispatch(int cfg, Fn&& fn) {
    switch (cfg) {
        case 0: fn(RefOps<C31>{}); return 0;
        case 1: fn(RefOps<C5>{}); return 0;
        case 2: fn(RefOps<CProt>{}); return 0;
        case 3: fn(RefOps<CTrip>{}); return 0;
        case 4: fn(RefOps<C31h8>{}); return 0;
        case 5: fn(RefOps<C31h16>{}); return 0;
        case 6: fn(RefOps<C21>{}); return 0;
        default: return -1;
    }
}

}  // namespace

extern "C" {

// Configuration ids: 0 = <31,28,16,4> DNA, 1 = <5,4,3,4> DNA, 2 = <5,4,3,4>
// protein, 3 = <3,2,2,4> DNA triplet, 4 = <31,28,16,8>, 5 = <31,28,16,16>,
// 6 = <21,19,11,4>.
int sbf_refcpu_insert(int cfg, const char* seq, uint64_t len, uint64_t* words,
                      uint64_t num_shards, int threads) {
    return dispatch(cfg, [&](auto ops) {
        using Ops = decltype(ops);
        Ops::insert_syms(Ops::encode(seq, len), false, words, num_shards, threads);
    });
}

int sbf_refcpu_contains(int cfg, const char* seq, uint64_t len, const uint64_t* words,
                        uint64_t num_shards, uint8_t* out, int threads) {
    return dispatch(cfg, [&](auto ops) {
        using Ops = decltype(ops);
        Ops::contains_syms(Ops::encode(seq, len), false, words, num_shards, out, threads);
    });
}

int sbf_refcpu_insert_dense(int cfg, const uint64_t* packed, uint64_t num_symbols,
                            uint64_t* words, uint64_t num_shards, int threads) {
    return dispatch(cfg, [&](auto ops) {
        using Ops = decltype(ops);
        Ops::insert_syms(Ops::decode_dense(packed, num_symbols), true, words, num_shards,
                         threads);
    });
}

int sbf_refcpu_contains_dense(int cfg, const uint64_t* packed, uint64_t num_symbols,
                              const uint64_t* words, uint64_t num_shards, uint8_t* out,
                              int threads) {
    return dispatch(cfg, [&](auto ops) {
        using Ops = decltype(ops);
        Ops::contains_syms(Ops::decode_dense(packed, num_symbols), true, words, num_shards, out,
                           threads);
    });
}
}
