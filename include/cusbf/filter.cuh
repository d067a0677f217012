// filter.cuh -- cusbf::filter<Config>, drop-in for the reference's
// include/cusbf/filter.cuh:68-1848 (tdortman/cuSBF) over libsbf_b200.
//
// Every member keeps the reference's name, signature, argument meaning and
// Result<T> error behaviour; each forwards to one entry point of the C ABI
// (include/sbf_b200.h) where the B200 kernels run.  *_async members do not
// synchronise the stream; the host-input members synchronise before
// returning.  Consumer exceptions propagate out of the query members and
// leave the filter usable, as in the reference.
//
// Link with libsbf_b200.so (cusbf_b200/libsbf_b200.so) and add include/ to
// the include path.
#pragma once

#include <cuda_runtime.h>

#include <cuda/stream_ref>

#include <exception>
#include <filesystem>
#include <istream>
#include <span>
#include <stdexcept>
#include <string>
#include <string_view>
#include <utility>
#include <vector>

#include <cusbf/Alphabet.cuh>
#include <cusbf/Fastx.hpp>
#include <cusbf/config.cuh>
#include <cusbf/cuda_error.hpp>
#include <cusbf/dense_packed.hpp>
#include <cusbf/device_span.cuh>
#include <cusbf/error.hpp>
#include <cusbf/filter_ref.cuh>
#include <cusbf/normalized_record_batch.hpp>

namespace cusbf {

namespace detail {

inline sbf_stream_t sbf_stream(cuda::stream_ref s) { return reinterpret_cast<sbf_stream_t>(s.get()); }

inline int64_t istream_read(void* user, char* buf, uint64_t cap) {
    auto* in = static_cast<std::istream*>(user);
    in->read(buf, static_cast<std::streamsize>(cap));
    const std::streamsize n = in->gcount();
    if (n == 0 && in->bad()) return -1;
    return static_cast<int64_t>(n);
}

template <typename Consumer>
struct RecordTrampoline {
    Consumer* consume;
    std::exception_ptr error;
    static int call(void* user, const sbf_record_view* v) {
        auto* t = static_cast<RecordTrampoline*>(user);
        try {
            (*t->consume)(RecordQueryView{
                v->record_index, std::string_view{v->sequence, v->sequence_bytes},
                v->queried_bases, v->queried_kmers, v->positive_kmers,
                std::span<const uint8_t>{v->hits, static_cast<size_t>(v->n_hits)}});
            return 0;
        } catch (...) {
            t->error = std::current_exception();
            return 1;
        }
    }
};

template <typename Consumer>
struct FastxTrampoline {
    Consumer* consume;
    std::exception_ptr error;
    static int call(void* user, const sbf_fastx_record_view* v) {
        auto* t = static_cast<FastxTrampoline*>(user);
        try {
            (*t->consume)(FastxRecordView{
                v->record_index, std::string_view{v->header, v->header_bytes},
                std::string_view{v->sequence, v->sequence_bytes}, v->queried_bases,
                v->queried_kmers, v->positive_kmers,
                std::span<const uint8_t>{v->hits, static_cast<size_t>(v->n_hits)}});
            return 0;
        } catch (...) {
            t->error = std::current_exception();
            return 1;
        }
    }
};

}  // namespace detail

template <typename Config>
class filter {
   public:
    using block_type = filter_block<Config>;
    using Shard = block_type;

    static_assert(Config::blockWordCount == 4, "Filter only supports the fused 256-bit shard path");

    explicit filter(uint64_t requestedFilterBits) {
        const int s = sbf_filter_create(Config::k, Config::s, Config::m,
                                        static_cast<uint32_t>(Config::hashCount),
                                        detail::alphabet_id<typename Config::Alphabet>(),
                                        requestedFilterBits, &handle_);
        if (s != SBF_OK) throw std::runtime_error(detail::status_error(s).message());
    }

    filter(const filter&) = delete;
    filter& operator=(const filter&) = delete;
    filter(filter&& other) noexcept : handle_(std::exchange(other.handle_, nullptr)) {}
    filter& operator=(filter&& other) noexcept {
        if (this != &other) {
            sbf_filter_destroy(handle_);
            handle_ = std::exchange(other.handle_, nullptr);
        }
        return *this;
    }
    ~filter() { sbf_filter_destroy(handle_); }

    [[nodiscard]] filter_ref<Config> ref() const noexcept {
        uint64_t* words = nullptr;
        uint64_t n = 0;
        sbf_filter_words(handle_, &words, &n);
        return filter_ref<Config>{reinterpret_cast<block_type*>(words), n / 4};
    }

    // ---- byte sequences (filter.cuh:154-190, :464-533) ----------------------
    [[nodiscard]] Result<uint64_t> insert_sequence(std::string_view sequence,
                                                   cuda::stream_ref stream = cudaStream_t{}) {
        uint64_t n = 0;
        const int s = sbf_insert_sequence(handle_, sequence.data(), sequence.size(),
                                          detail::sbf_stream(stream), &n);
        if (s != SBF_OK) return Err(detail::status_error(s));
        return n;
    }

    [[nodiscard]] Result<uint64_t> insert_sequence_async(device_span<const char> d_sequence,
                                                         cuda::stream_ref stream = cudaStream_t{}) {
        uint64_t n = 0;
        const int s = sbf_insert_sequence_async(handle_, d_sequence.data(), d_sequence.size(),
                                                detail::sbf_stream(stream), &n);
        if (s != SBF_OK) return Err(detail::status_error(s));
        return n;
    }

    [[nodiscard]] Result<void> contains_sequence_async(device_span<const char> d_sequence,
                                                       device_span<uint8_t> d_output,
                                                       cuda::stream_ref stream = cudaStream_t{}) const {
        const int s = sbf_contains_sequence_async(handle_, d_sequence.data(), d_sequence.size(),
                                                  d_output.data(), d_output.size(),
                                                  detail::sbf_stream(stream));
        if (s != SBF_OK) return Err(detail::status_error(s));
        return {};
    }

    [[nodiscard]] Result<void> contains_sequence(std::string_view sequence,
                                                 device_span<uint8_t> d_output,
                                                 cuda::stream_ref stream = cudaStream_t{}) const {
        const int s = sbf_contains_sequence_to_device(handle_, sequence.data(), sequence.size(),
                                                      d_output.data(), d_output.size(),
                                                      detail::sbf_stream(stream));
        if (s != SBF_OK) return Err(detail::status_error(s));
        return {};
    }

    [[nodiscard]] Result<std::vector<uint8_t>> contains_sequence(
        std::string_view sequence, cuda::stream_ref stream = cudaStream_t{}) const {
        std::vector<uint8_t> out(sbf_filter_kmer_count(handle_, sequence.size()));
        if (out.empty()) return out;
        const int s = sbf_contains_sequence(handle_, sequence.data(), sequence.size(), out.data(),
                                            out.size(), detail::sbf_stream(stream));
        if (s != SBF_OK) return Err(detail::status_error(s));
        return out;
    }

    // ---- dense packed input (filter.cuh:207-322) -----------------------------
    [[nodiscard]] Result<uint64_t> insert_dense_packed_async(device_span<const uint64_t> d_words,
                                                             uint64_t num_symbols,
                                                             cuda::stream_ref stream = cudaStream_t{}) {
        uint64_t n = 0;
        const int s = sbf_insert_dense_packed_async(handle_, d_words.data(), d_words.size(),
                                                    num_symbols, detail::sbf_stream(stream), &n);
        if (s != SBF_OK) return Err(detail::status_error(s));
        return n;
    }

    [[nodiscard]] Result<uint64_t> insert_dense_packed(std::span<const uint64_t> words,
                                                       uint64_t num_symbols,
                                                       cuda::stream_ref stream = cudaStream_t{}) {
        uint64_t n = 0;
        const int s = sbf_insert_dense_packed(handle_, words.data(), words.size(), num_symbols,
                                              detail::sbf_stream(stream), &n);
        if (s != SBF_OK) return Err(detail::status_error(s));
        return n;
    }

    [[nodiscard]] Result<void> contains_dense_packed_async(device_span<const uint64_t> d_words,
                                                           uint64_t num_symbols,
                                                           device_span<uint8_t> d_output,
                                                           cuda::stream_ref stream = cudaStream_t{}) const {
        const int s = sbf_contains_dense_packed_async(handle_, d_words.data(), d_words.size(),
                                                      num_symbols, d_output.data(),
                                                      d_output.size(), detail::sbf_stream(stream));
        if (s != SBF_OK) return Err(detail::status_error(s));
        return {};
    }

    [[nodiscard]] Result<void> contains_dense_packed(std::span<const uint64_t> words,
                                                     uint64_t num_symbols,
                                                     device_span<uint8_t> d_output,
                                                     cuda::stream_ref stream = cudaStream_t{}) const {
        const int s = sbf_contains_dense_packed_to_device(handle_, words.data(), words.size(),
                                                          num_symbols, d_output.data(),
                                                          d_output.size(), detail::sbf_stream(stream));
        if (s != SBF_OK) return Err(detail::status_error(s));
        return {};
    }

    [[nodiscard]] Result<std::vector<uint8_t>> contains_dense_packed(
        std::span<const uint64_t> words, uint64_t num_symbols,
        cuda::stream_ref stream = cudaStream_t{}) const {
        std::vector<uint8_t> out(dense_packed_kmer_count(num_symbols));
        if (out.empty()) return out;
        const int s = sbf_contains_dense_packed(handle_, words.data(), words.size(), num_symbols,
                                                out.data(), out.size(), detail::sbf_stream(stream));
        if (s != SBF_OK) return Err(detail::status_error(s));
        return out;
    }

    [[nodiscard]] static constexpr uint64_t dense_packed_word_count(uint64_t num_symbols) {
        return cusbf::dense_packed_word_count<Config>(num_symbols);
    }
    [[nodiscard]] constexpr uint64_t dense_packed_kmer_count(uint64_t num_symbols) const {
        return cusbf::dense_packed_kmer_count<Config>(num_symbols);
    }

    // ---- record batches (filter.cuh:338-400, :549-622) -----------------------
    [[nodiscard]] Result<FastxInsertReport> insert_record_batch(
        RecordBatchView batch, cuda::stream_ref stream = cudaStream_t{}) {
        FastxInsertReport rep{};
        const int s = sbf_insert_record_batch(
            handle_, batch.sequence.data(), batch.sequence.size(),
            reinterpret_cast<const sbf_record_range*>(batch.records.data()), batch.records.size(),
            detail::sbf_stream(stream), reinterpret_cast<sbf_insert_report*>(&rep));
        if (s != SBF_OK) return Err(detail::status_error(s));
        return rep;
    }

    [[nodiscard]] Result<uint64_t> insert_record_batch_async(
        device_span<const char> d_sequence, std::span<const RecordRange> records,
        cuda::stream_ref stream = cudaStream_t{}) {
        uint64_t n = 0;
        const int s = sbf_insert_record_batch_async(
            handle_, d_sequence.data(), d_sequence.size(),
            reinterpret_cast<const sbf_record_range*>(records.data()), records.size(),
            detail::sbf_stream(stream), &n);
        if (s != SBF_OK) return Err(detail::status_error(s));
        return n;
    }

    [[nodiscard]] Result<FastxQueryReport> query_record_batch(
        RecordBatchView batch, cuda::stream_ref stream = cudaStream_t{}) const {
        FastxQueryReport rep{};
        const int s = sbf_query_record_batch(
            handle_, batch.sequence.data(), batch.sequence.size(),
            reinterpret_cast<const sbf_record_range*>(batch.records.data()), batch.records.size(),
            detail::sbf_stream(stream), reinterpret_cast<sbf_query_report*>(&rep), nullptr, nullptr);
        if (s != SBF_OK) return Err(detail::status_error(s));
        return rep;
    }

    template <RecordQueryConsumer Consumer>
    [[nodiscard]] Result<FastxQueryReport> query_record_batch(
        RecordBatchView batch, Consumer&& consume, cuda::stream_ref stream = cudaStream_t{}) const {
        FastxQueryReport rep{};
        using C = std::remove_reference_t<Consumer>;
        detail::RecordTrampoline<C> t{&consume, nullptr};
        const int s = sbf_query_record_batch(
            handle_, batch.sequence.data(), batch.sequence.size(),
            reinterpret_cast<const sbf_record_range*>(batch.records.data()), batch.records.size(),
            detail::sbf_stream(stream), reinterpret_cast<sbf_query_report*>(&rep),
            &detail::RecordTrampoline<C>::call, &t);
        if (t.error) std::rethrow_exception(t.error);
        if (s != SBF_OK) return Err(detail::status_error(s));
        return rep;
    }

    [[nodiscard]] Result<void> contains_record_batch_async(
        device_span<const char> d_sequence, std::span<const RecordRange> records,
        device_span<uint8_t> d_output, cuda::stream_ref stream = cudaStream_t{}) const {
        const int s = sbf_contains_record_batch_async(
            handle_, d_sequence.data(), d_sequence.size(),
            reinterpret_cast<const sbf_record_range*>(records.data()), records.size(),
            d_output.data(), d_output.size(), detail::sbf_stream(stream));
        if (s != SBF_OK) return Err(detail::status_error(s));
        return {};
    }

    // ---- FASTA / FASTQ (filter.cuh:416-452, :632-786) ------------------------
    [[nodiscard]] Result<FastxInsertReport> insert_fastx(std::istream& input,
                                                         double fill_fraction = 0.7,
                                                         cuda::stream_ref stream = cudaStream_t{}) {
        FastxInsertReport rep{};
        const int s = sbf_insert_fastx(handle_, &detail::istream_read, &input, "<stream>",
                                       fill_fraction, detail::sbf_stream(stream),
                                       reinterpret_cast<sbf_insert_report*>(&rep));
        if (s != SBF_OK) return Err(detail::status_error(s));
        return rep;
    }

    [[nodiscard]] Result<FastxInsertReport> insert_fastx_file(
        const std::filesystem::path& path, double fill_fraction = 0.7,
        cuda::stream_ref stream = cudaStream_t{}) {
        FastxInsertReport rep{};
        const int s = sbf_insert_fastx_file(handle_, path.c_str(), fill_fraction,
                                            detail::sbf_stream(stream),
                                            reinterpret_cast<sbf_insert_report*>(&rep));
        if (s != SBF_OK) return Err(detail::status_error(s));
        return rep;
    }

    [[nodiscard]] Result<FastxQueryReport> query_fastx(std::istream& input,
                                                       double fill_fraction = 0.7,
                                                       cuda::stream_ref stream = cudaStream_t{}) const {
        FastxQueryReport rep{};
        const int s = sbf_query_fastx(handle_, &detail::istream_read, &input, "<stream>",
                                      fill_fraction, detail::sbf_stream(stream),
                                      reinterpret_cast<sbf_query_report*>(&rep), nullptr, nullptr);
        if (s != SBF_OK) return Err(detail::status_error(s));
        return rep;
    }

    [[nodiscard]] Result<FastxQueryReport> query_fastx_file(
        const std::filesystem::path& path, double fill_fraction = 0.7,
        cuda::stream_ref stream = cudaStream_t{}) const {
        FastxQueryReport rep{};
        const int s = sbf_query_fastx_file(handle_, path.c_str(), fill_fraction,
                                           detail::sbf_stream(stream),
                                           reinterpret_cast<sbf_query_report*>(&rep), nullptr,
                                           nullptr);
        if (s != SBF_OK) return Err(detail::status_error(s));
        return rep;
    }

    template <FastxRecordConsumer Consumer>
    [[nodiscard]] Result<FastxQueryReport> query_fastx_records(
        std::istream& input, Consumer&& consume, double fill_fraction = 0.7,
        cuda::stream_ref stream = cudaStream_t{}) const {
        FastxQueryReport rep{};
        using C = std::remove_reference_t<Consumer>;
        detail::FastxTrampoline<C> t{&consume, nullptr};
        const int s = sbf_query_fastx(handle_, &detail::istream_read, &input, "<stream>",
                                      fill_fraction, detail::sbf_stream(stream),
                                      reinterpret_cast<sbf_query_report*>(&rep),
                                      &detail::FastxTrampoline<C>::call, &t);
        if (t.error) std::rethrow_exception(t.error);
        if (s != SBF_OK) return Err(detail::status_error(s));
        return rep;
    }

    template <FastxRecordConsumer Consumer>
    [[nodiscard]] Result<FastxQueryReport> query_fastx_file_records(
        const std::filesystem::path& path, Consumer&& consume, double fill_fraction = 0.7,
        cuda::stream_ref stream = cudaStream_t{}) const {
        FastxQueryReport rep{};
        using C = std::remove_reference_t<Consumer>;
        detail::FastxTrampoline<C> t{&consume, nullptr};
        const int s = sbf_query_fastx_file(handle_, path.c_str(), fill_fraction,
                                           detail::sbf_stream(stream),
                                           reinterpret_cast<sbf_query_report*>(&rep),
                                           &detail::FastxTrampoline<C>::call, &t);
        if (t.error) std::rethrow_exception(t.error);
        if (s != SBF_OK) return Err(detail::status_error(s));
        return rep;
    }

    [[nodiscard]] Result<FastxDetailedQueryReport> query_fastx_detailed(
        std::istream& input, double fill_fraction = 0.7,
        cuda::stream_ref stream = cudaStream_t{}) const {
        FastxDetailedQueryReport report;
        auto keep = [&report](const FastxRecordView& r) { report.records.push_back(owned(r)); };
        report.summary = CUSBF_TRY(query_fastx_records(input, keep, fill_fraction, stream));
        return report;
    }

    [[nodiscard]] Result<FastxDetailedQueryReport> query_fastx_file_detailed(
        const std::filesystem::path& path, double fill_fraction = 0.7,
        cuda::stream_ref stream = cudaStream_t{}) const {
        FastxDetailedQueryReport report;
        auto keep = [&report](const FastxRecordView& r) { report.records.push_back(owned(r)); };
        report.summary = CUSBF_TRY(query_fastx_file_records(path, keep, fill_fraction, stream));
        return report;
    }

    // ---- state (filter.cuh:793-833) -------------------------------------------
    [[nodiscard]] Result<void> clear(cuda::stream_ref stream = cudaStream_t{}) {
        const int s = sbf_filter_clear(handle_, detail::sbf_stream(stream));
        if (s != SBF_OK) return Err(detail::status_error(s));
        return {};
    }

    [[nodiscard]] float load_factor() const {
        double lf = 0;
        const int s = sbf_filter_load_factor(handle_, nullptr, &lf);
        if (s != SBF_OK) throw std::runtime_error(detail::status_error(s).message());
        return static_cast<float>(lf);
    }

    [[nodiscard]] uint64_t filter_bits() const { return sbf_filter_bits(handle_); }
    [[nodiscard]] uint64_t num_shards() const { return sbf_filter_num_shards(handle_); }

    // The C-ABI handle (for callers mixing the C and C++ interfaces).
    [[nodiscard]] sbf_filter_t* handle() const noexcept { return handle_; }

   private:
    static FastxDetailedQueryRecord owned(const FastxRecordView& r) {
        return FastxDetailedQueryRecord{r.record_index,        std::string(r.header),
                                        std::string(r.sequence), r.queriedBases,
                                        r.queriedKmers,        r.positive_kmers,
                                        std::vector<uint8_t>(r.hits.begin(), r.hits.end())};
    }

    sbf_filter_t* handle_ = nullptr;
};

}  // namespace cusbf
