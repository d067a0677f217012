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
class ExpandPool {
public:
    explicit ExpandPool(int threads);
    ~ExpandPool();
    ExpandPool(const ExpandPool&) = delete;
    ExpandPool& operator=(const ExpandPool&) = delete;
    void run(const uint32_t* bits, uint8_t* out, uint64_t n);  // returns when done

private:
    struct Job {
        const uint32_t* bits = nullptr;
        uint64_t j0 = 0;          // window of the first block
        uint8_t* body = nullptr;  // 32-byte aligned
        uint64_t blocks = 0;
    };
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
