// query_layout.cuh -- per-record hit spans of a normalised batch (drop-in for
// the reference's include/cusbf/detail/query_layout.cuh:13-72), implemented
// by sbf_query_layout of libsbf_b200.
#pragma once

#include <span>
#include <vector>

#include <cusbf/normalized_record_batch.hpp>

namespace cusbf::detail {

struct QueryLayoutRecord {
    uint64_t record_index{};
    uint64_t input_offset{};
    uint64_t size{};
    uint64_t valid_kmers{};
    uint64_t hit_offset{};
    uint64_t hit_count{};
};
static_assert(sizeof(QueryLayoutRecord) == sizeof(sbf_query_layout_record));

class QueryLayout {
   public:
    [[nodiscard]] std::span<const QueryLayoutRecord> records() const noexcept {
        return {records_.data(), records_.size()};
    }
    [[nodiscard]] uint64_t total_hit_count() const noexcept { return total_hit_count_; }
    [[nodiscard]] std::span<const uint8_t> hits_for_record(std::span<const uint8_t> hits,
                                                           size_t layout_index) const noexcept {
        const QueryLayoutRecord& r = records_[layout_index];
        return {hits.data() + r.hit_offset, static_cast<size_t>(r.hit_count)};
    }
    template <typename Config>
    [[nodiscard]] static QueryLayout build(std::span<const NormalizedRecord> records) {
        QueryLayout layout;
        layout.records_.resize(records.size());
        sbf_query_layout_for(detail::alphabet_id<typename Config::Alphabet>(), Config::k,
                             reinterpret_cast<const sbf_normalized_record*>(records.data()),
                             records.size(),
                             reinterpret_cast<sbf_query_layout_record*>(layout.records_.data()),
                             &layout.total_hit_count_);
        return layout;
    }

   private:
    std::vector<QueryLayoutRecord> records_{};
    uint64_t total_hit_count_{};
};

}  // namespace cusbf::detail
