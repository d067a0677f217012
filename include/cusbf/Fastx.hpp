// Fastx.hpp -- record batches and FASTX result types (drop-in for the
// reference's include/cusbf/Fastx.hpp:24-238).  Parsing itself lives in
// libsbf_b200 (sbf_fastx_scan and the FASTX entry points of sbf_b200.h).
#pragma once

#include <cassert>
#include <concepts>
#include <cstdint>
#include <span>
#include <string>
#include <string_view>
#include <vector>

#include <cusbf/error.hpp>

namespace cusbf {

struct RecordRange {
    uint64_t sequenceOffset{};
    uint64_t sequenceBytes{};
};
static_assert(sizeof(RecordRange) == sizeof(sbf_record_range));

struct RecordBatchView {
    std::string_view sequence{};
    std::span<const RecordRange> records{};
};

class DenseRecordBatchBuilder {
   public:
    explicit DenseRecordBatchBuilder(uint64_t reserve_bytes = 0) {
        if (reserve_bytes) sequence_.reserve(static_cast<size_t>(reserve_bytes));
    }
    [[nodiscard]] std::string_view sequence_view() const noexcept {
        return external_sequence_.empty() ? std::string_view{sequence_} : external_sequence_;
    }
    [[nodiscard]] RecordBatchView view() const noexcept {
        return RecordBatchView{sequence_view(), {ranges_.data(), ranges_.size()}};
    }
    void appendRecord(std::string_view record_sequence) {
        assert(external_sequence_.empty());
        ranges_.push_back(RecordRange{sequence_.size(), record_sequence.size()});
        sequence_.append(record_sequence);
    }
    void push_range(RecordRange range) { ranges_.push_back(range); }
    [[nodiscard]] std::string& sequence_buffer() noexcept { return sequence_; }
    [[nodiscard]] std::string_view& external_sequence_slot() noexcept { return external_sequence_; }
    [[nodiscard]] bool empty() const noexcept { return ranges_.empty(); }
    [[nodiscard]] uint64_t recordCount() const noexcept { return ranges_.size(); }
    [[nodiscard]] uint64_t raw_sequence_bytes() const noexcept {
        if (external_sequence_.empty()) return sequence_.size();
        uint64_t total = 0;
        for (const RecordRange& r : ranges_) total += r.sequenceBytes;
        return total;
    }
    [[nodiscard]] const std::vector<RecordRange>& ranges() const noexcept { return ranges_; }
    void clear() {
        sequence_.clear();
        ranges_.clear();
        external_sequence_ = {};
    }
    void clear_and_shrink() {
        clear();
        std::string{}.swap(sequence_);
        std::vector<RecordRange>{}.swap(ranges_);
    }

   private:
    std::string sequence_;
    std::string_view external_sequence_{};
    std::vector<RecordRange> ranges_;
};

struct RecordQueryView {
    uint64_t record_index{};
    std::string_view sequence{};
    uint64_t queriedBases{};
    uint64_t queriedKmers{};
    uint64_t positive_kmers{};
    std::span<const uint8_t> hits{};
};

struct FastxInsertReport {
    uint64_t recordsIndexed{};
    uint64_t indexedBases{};
    uint64_t insertedKmers{};
};
static_assert(sizeof(FastxInsertReport) == sizeof(sbf_insert_report));

struct FastxQueryReport {
    uint64_t recordsQueried{};
    uint64_t queriedBases{};
    uint64_t queriedKmers{};
    uint64_t positive_kmers{};
};
static_assert(sizeof(FastxQueryReport) == sizeof(sbf_query_report));

struct FastxRecordView {
    uint64_t record_index{};
    std::string_view header{};
    std::string_view sequence{};
    uint64_t queriedBases{};
    uint64_t queriedKmers{};
    uint64_t positive_kmers{};
    std::span<const uint8_t> hits{};
};

struct FastxDetailedQueryRecord {
    uint64_t record_index{};
    std::string header;
    std::string sequence;
    uint64_t queriedBases{};
    uint64_t queriedKmers{};
    uint64_t positive_kmers{};
    std::vector<uint8_t> hits;
};

struct FastxDetailedQueryReport {
    FastxQueryReport summary{};
    std::vector<FastxDetailedQueryRecord> records;
};

template <typename Functor>
concept RecordQueryConsumer = requires(Functor f, const RecordQueryView& view) {
    { f(view) } -> std::same_as<void>;
};

template <typename Functor>
concept FastxRecordConsumer = requires(Functor f, const FastxRecordView& record) {
    { f(record) } -> std::same_as<void>;
};

}  // namespace cusbf
