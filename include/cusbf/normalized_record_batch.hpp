// normalized_record_batch.hpp -- separator-joined record batches (drop-in for
// the reference's include/cusbf/normalized_record_batch.hpp:20-316),
// implemented by sbf_normalize_record_batch of libsbf_b200.
#pragma once

#include <span>
#include <string>
#include <vector>

#include <cusbf/Fastx.hpp>
#include <cusbf/config.cuh>
#include <cusbf/error.hpp>

namespace cusbf {

struct NormalizedRecord {
    uint64_t record_index{};
    uint64_t input_offset{};
    uint64_t size{};
    uint64_t valid_kmers{};
};
static_assert(sizeof(NormalizedRecord) == sizeof(sbf_normalized_record));

template <typename Config>
[[nodiscard]] Result<void> normalize_record_batch_into(RecordBatchView batch,
                                                       std::string& sequence_out,
                                                       std::vector<NormalizedRecord>& records_out) {
    constexpr int alphabet = detail::alphabet_id<typename Config::Alphabet>();
    const auto* r = reinterpret_cast<const sbf_record_range*>(batch.records.data());
    const uint64_t n = batch.records.size();
    uint64_t total = 0;
    int s = sbf_normalize_record_batch_for(alphabet, Config::k, batch.sequence.data(),
                                           batch.sequence.size(), r, n, nullptr, 0, &total,
                                           nullptr);
    if (s != SBF_OK) return Err(detail::status_error(s));
    sequence_out.resize(total);
    records_out.resize(n);
    s = sbf_normalize_record_batch_for(
        alphabet, Config::k, batch.sequence.data(), batch.sequence.size(), r, n,
        sequence_out.data(), total, &total,
        reinterpret_cast<sbf_normalized_record*>(records_out.data()));
    if (s != SBF_OK) return Err(detail::status_error(s));
    return {};
}

class NormalizedRecordBatch {
   public:
    [[nodiscard]] const std::string& sequence() const noexcept { return sequence_; }
    [[nodiscard]] std::span<const NormalizedRecord> records() const noexcept {
        return {records_.data(), records_.size()};
    }
    [[nodiscard]] uint64_t total_valid_kmers() const noexcept {
        uint64_t total = 0;
        for (const NormalizedRecord& r : records_) total += r.valid_kmers;
        return total;
    }

   private:
    template <typename Config>
    friend Result<NormalizedRecordBatch> normalize_record_batch(RecordBatchView batch);
    std::string sequence_;
    std::vector<NormalizedRecord> records_;
};

template <typename Config>
[[nodiscard]] Result<NormalizedRecordBatch> normalize_record_batch(RecordBatchView batch) {
    NormalizedRecordBatch out;
    CUSBF_TRY(normalize_record_batch_into<Config>(batch, out.sequence_, out.records_));
    return out;
}

}  // namespace cusbf
