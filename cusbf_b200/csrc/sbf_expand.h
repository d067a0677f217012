// sbf_expand.h -- host expansion of bit-packed query results into bytes.
#pragma once

#include <condition_variable>
#include <cstdint>
#include <mutex>
#include <thread>
#include <vector>

namespace sbf {

// A fixed pool of host threads (the caller counts as one) that writes
// out[i] = bit i % 32 of bits[i / 32] for i < n; it reads only the words
// that hold those bits.
// One expansion: out[i] = bit i of `bits` for i < n.
struct ExpandItem {
    const uint32_t* bits;
    uint8_t* out;
    uint64_t n;
};

class ExpandPool {
public:
    explicit ExpandPool(int threads);
    ~ExpandPool();
    ExpandPool(const ExpandPool&) = delete;
    ExpandPool& operator=(const ExpandPool&) = delete;
    void run(const uint32_t* bits, uint8_t* out, uint64_t n);  // returns when done
    // Many expansions (one per served request), each on one thread.
    void run_items(const ExpandItem* items, size_t n_items);

private:
    struct Job {
        const uint32_t* bits = nullptr;
        uint64_t j0 = 0;          // window of the first block
        uint8_t* body = nullptr;  // 32-byte aligned
        uint64_t blocks = 0;
        const ExpandItem* items = nullptr;  // run_items: the list, else null
        size_t n_items = 0;
    };
    void dispatch();  // runs job_ on every thread, returns when all are done
    void worker(int t);
    void part(int t, int parts);

    int threads_;
    Job job_;
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_cv_;
    uint64_t gen_ = 0;
    int pending_ = 0;
    bool stop_ = false;
};

// Threads to expand host query results with (0: download bytes instead).
int host_expand_threads();

}  // namespace sbf
