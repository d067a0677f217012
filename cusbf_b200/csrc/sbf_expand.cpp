// sbf_expand.cpp -- host expansion of bit-packed query results (window i ->
// bit i % 32 of word i / 32) into one byte per window (0 or 1), the layout
// of contains_sequence's host output (include/cusbf/filter.cuh:514).
//
// Host-output queries download one bit per window, an eighth of the bytes,
// and a pool of host threads writes the bytes while later chunks upload.
// Each 32-window word becomes 32 output bytes: AVX2 broadcasts the word,
// routes byte i / 8 of it to output byte i, tests bit i % 8 and keeps 0/1,
// and writes whole 32-byte lines with streaming stores.  Hosts without AVX2
// use a 256-entry table of 8-byte patterns.
#include <immintrin.h>

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/sbf_b200.h"
#include "sbf_expand.h"
#include "sbf_host.h"

namespace sbf {
namespace {

struct Lut {
    uint64_t v[256];
    Lut() {
        for (int b = 0; b < 256; ++b) {
            uint64_t x = 0;
            for (int i = 0; i < 8; ++i) x |= static_cast<uint64_t>((b >> i) & 1) << (8 * i);
            v[b] = x;
        }
    }
};
const Lut g_lut;

inline uint8_t bit_at(const uint32_t* bits, uint64_t i) {
    return static_cast<uint8_t>((bits[i >> 5] >> (i & 31)) & 1u);
}

// The 32 bits of windows j .. j+31, for j + 31 < n (j need not be a
// multiple of 32: the word after j / 32 then holds window j + 31).
inline uint32_t bits_from(const uint32_t* bits, uint64_t j) {
    const uint32_t s = static_cast<uint32_t>(j & 31);
    const uint64_t w = j >> 5;
    if (s == 0) return bits[w];
    return static_cast<uint32_t>(
        ((static_cast<uint64_t>(bits[w + 1]) << 32) | bits[w]) >> s);
}

// Blocks [b0, b1) of 32 windows starting at window j0 + 32 * b, written to
// out + 32 * b (32-byte aligned).
void blocks_scalar(const uint32_t* bits, uint64_t j0, uint8_t* out, uint64_t b0, uint64_t b1) {
    for (uint64_t b = b0; b < b1; ++b) {
        const uint32_t x = bits_from(bits, j0 + 32 * b);
        uint64_t q[4];
        for (int k = 0; k < 4; ++k) q[k] = g_lut.v[(x >> (8 * k)) & 0xFFu];
        std::memcpy(out + 32 * b, q, 32);
    }
}

__attribute__((target("avx2"))) void blocks_avx2(const uint32_t* bits, uint64_t j0, uint8_t* out,
                                                 uint64_t b0, uint64_t b1) {
    const __m256i route = _mm256_setr_epi8(0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 2, 2,
                                           2, 2, 2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 3, 3);
    const __m256i probe = _mm256_set1_epi64x(static_cast<long long>(0x8040201008040201ull));
    const __m256i one = _mm256_set1_epi8(1);
    for (uint64_t b = b0; b < b1; ++b) {
        __m256i v = _mm256_set1_epi32(static_cast<int>(bits_from(bits, j0 + 32 * b)));
        v = _mm256_shuffle_epi8(v, route);
        v = _mm256_and_si256(_mm256_cmpeq_epi8(_mm256_and_si256(v, probe), probe), one);
        _mm256_stream_si256(reinterpret_cast<__m256i*>(out + 32 * b), v);
    }
    _mm_sfence();
}

bool have_avx2() {
    static const bool yes = __builtin_cpu_supports("avx2");
    return yes;
}

void blocks_any(const uint32_t* bits, uint64_t j0, uint8_t* out, uint64_t b0, uint64_t b1) {
    if (have_avx2())
        blocks_avx2(bits, j0, out, b0, b1);
    else
        blocks_scalar(bits, j0, out, b0, b1);
}

// Head bytes up to the first 32-byte boundary of `out`, whole 32-window
// blocks after it, and the tail; returns the head length and block count.
void split(const uint8_t* out, uint64_t n, uint64_t* head, uint64_t* blocks) {
    *head = std::min<uint64_t>(n, (32 - (reinterpret_cast<uintptr_t>(out) & 31u)) & 31u);
    *blocks = (n - *head) / 32;
}

void edges(const uint32_t* bits, uint8_t* out, uint64_t n, uint64_t head, uint64_t blocks) {
    for (uint64_t i = 0; i < head; ++i) out[i] = bit_at(bits, i);
    for (uint64_t i = head + 32 * blocks; i < n; ++i) out[i] = bit_at(bits, i);
}

void expand_serial(const ExpandItem& it) {
    uint64_t head, blocks;
    split(it.out, it.n, &head, &blocks);
    edges(it.bits, it.out, it.n, head, blocks);
    if (blocks) blocks_any(it.bits, head, it.out + head, 0, blocks);
}

}  // namespace

ExpandPool::ExpandPool(int threads) : threads_(std::max(threads, 1)) {
    try {
        for (int t = 1; t < threads_; ++t) workers_.emplace_back([this, t] { worker(t); });
    } catch (...) {
        // Stop the workers that did start, then report the failure.
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& w : workers_) w.join();
        throw;
    }
}

ExpandPool::~ExpandPool() {
    {
        std::lock_guard<std::mutex> g(m_);
        stop_ = true;
    }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
}

void ExpandPool::part(int t, int parts) {
    if (job_.items) {
        for (size_t i = static_cast<size_t>(t); i < job_.n_items; i += static_cast<size_t>(parts))
            expand_serial(job_.items[i]);
        return;
    }
    const uint64_t lo = job_.blocks * static_cast<uint64_t>(t) / parts;
    const uint64_t hi = job_.blocks * static_cast<uint64_t>(t + 1) / parts;
    if (lo < hi) blocks_any(job_.bits, job_.j0, job_.body, lo, hi);
}

void ExpandPool::dispatch() {
    {
        std::lock_guard<std::mutex> g(m_);
        pending_ = threads_ - 1;
        ++gen_;
    }
    cv_.notify_all();
    part(0, threads_);
    std::unique_lock<std::mutex> l(m_);
    done_cv_.wait(l, [&] { return pending_ == 0; });
}

void ExpandPool::worker(int t) {
    uint64_t seen = 0;
    for (;;) {
        {
            std::unique_lock<std::mutex> l(m_);
            cv_.wait(l, [&] { return stop_ || gen_ != seen; });
            if (stop_) return;
            seen = gen_;
        }
        part(t, threads_);
        {
            std::lock_guard<std::mutex> g(m_);
            if (--pending_ == 0) done_cv_.notify_one();
        }
    }
}

void ExpandPool::run(const uint32_t* bits, uint8_t* out, uint64_t n) {
    if (n == 0) return;
    uint64_t head, blocks;
    split(out, n, &head, &blocks);
    edges(bits, out, n, head, blocks);
    if (blocks == 0) return;
    job_ = Job{bits, head, out + head, blocks, nullptr, 0};
    // Small jobs are not worth waking the pool.
    if (threads_ == 1 || blocks < 4096) {
        part(0, 1);
        return;
    }
    dispatch();
}

void ExpandPool::run_items(const ExpandItem* items, size_t n_items) {
    if (n_items == 0) return;
    if (n_items == 1) {
        run(items[0].bits, items[0].out, items[0].n);
        return;
    }
    uint64_t total = 0;
    for (size_t i = 0; i < n_items; ++i) total += items[i].n;
    job_ = Job{};
    job_.items = items;
    job_.n_items = n_items;
    if (threads_ == 1 || total < 32 * 4096) {
        part(0, 1);
        return;
    }
    dispatch();
}

int host_expand_threads() {
    // SBF_HOST_EXPAND=0 keeps byte downloads; =1 forces expansion; unset:
    // expand on hosts with at least 8 hardware threads.  Four threads (or
    // SBF_HOST_EXPAND_THREADS): on a 16-thread B200 host the 15 GB query of
    // 100M reads returned its bytes at 51 GB/s with 4 threads, 46 with 8,
    // 32 with 15 (the writes compete with the uploads for host memory), and
    // 48 GB/s when downloading bytes.
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    int want = static_cast<int>(std::min(4u, std::max(1u, hw / 2)));
    if (const char* v = std::getenv("SBF_HOST_EXPAND_THREADS")) {
        const long t = std::strtol(v, nullptr, 10);
        if (t > 0) want = static_cast<int>(std::min<long>(t, 64));
    }
    if (const char* v = std::getenv("SBF_HOST_EXPAND")) {
        if (v[0] == '0') return 0;
        if (v[0] == '1') return want;
    }
    return hw >= 8 ? want : 0;
}

}  // namespace sbf

extern "C" int sbf_expand_result_bits(const uint32_t* bits, uint64_t n_windows, uint8_t* out,
                                      uint32_t threads) {
    if (n_windows == 0) return SBF_OK;
    if (!bits || !out) return sbf::set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int t = threads ? static_cast<int>(std::min(threads, 64u))
                          : static_cast<int>(std::min(4u, std::max(1u, hw / 2)));
    try {
        sbf::ExpandPool pool(t);
        pool.run(bits, out, n_windows);
    } catch (...) {
        return sbf::set_error(SBF_ERR_RESOURCE, "cannot start host expansion threads");
    }
    return SBF_OK;
}

extern "C" int sbf_host_expand_threads(void) { return sbf::host_expand_threads(); }
