// sbf_host.h -- host-side filter object behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/sbf_b200.h"
#include "sbf_internal.h"

namespace sbf {

int set_error(int status, const char* fmt, ...);
// Bits per packed symbol and input bytes per symbol of an alphabet
// (SBF_ALPHABET_*); false for an unknown alphabet (sbf_generic.cu).
bool alphabet_geometry(int alphabet, uint32_t* bits, uint32_t* width);
void set_error_location(const char* file, uint32_t line, uint32_t col);
int cuda_fail(cudaError_t e, const char* what);
bool is_pinned(const void* p);

// A pair of device buffers and a pair of pinned host buffers, grown on
// demand and reused across calls.
// Chunks of a host-input call in flight at once (upload, kernel, download).
constexpr int kPipeSlots = 3;

struct Staging {
    void* dev[kPipeSlots] = {};
    void* pin[kPipeSlots] = {};
    size_t dev_cap = 0;
    size_t pin_cap = 0;
    int ensure_device(size_t bytes);
    int ensure_pinned(size_t bytes);
    void release();
};

// A grow-only pinned host buffer.
struct PinnedBuf {
    void* p = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes);
    void release();
};

// A grow-only device buffer.
struct DevBuf {
    void* ptr = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes);
    void release();
};

struct RaggedState;
struct FastqDevice;
class ExpandPool;

}  // namespace sbf

struct sbf_filter {
    const sbf::KernelSet* ks = nullptr;
    uint32_t k = 0, s = 0, m = 0, h = 0;
    int alphabet = 0;
    uint32_t width = 1;  // input bytes per symbol (3 for DNA triplets)
    sbf::GenericCfg gen{};
    uint64_t num_shards = 0;
    uint64_t filter_bits = 0;
    uint64_t* d_words = nullptr;
    int* d_err = nullptr;  // [0] device error word, [8..9] popcount scratch
    int device = 0;
    int sms = 0;
    int occupancy[6] = {1, 1, 1, 1, 1, 1};  // insert/query x bytes/dense/ragged
    mutable uint64_t launches = 0;

    sbf::Staging stage_in;
    sbf::Staging stage_out;
    cudaStream_t copy_stream = nullptr;  // host -> device chunk uploads
    cudaStream_t d2h_stream = nullptr;   // device -> host result downloads
    cudaEvent_t ev_copied[sbf::kPipeSlots] = {};
    cudaEvent_t ev_kernel[sbf::kPipeSlots] = {};
    cudaEvent_t ev_done[sbf::kPipeSlots] = {};

    // Ragged-batch engine state (sbf_ragged.cu), created on first use.
    sbf::RaggedState* ragged = nullptr;
    // FASTQ device parser buffers (sbf_fastq_gpu.cu), created on first use,
    // and the pinned block of input text it parses.
    sbf::FastqDevice* fastq = nullptr;
    sbf::PinnedBuf fastq_block;
    // The second block buffer of FASTQ input read ahead while the device
    // processes the current block.
    sbf::PinnedBuf fastq_ahead;

    // Record-batch staging (sbf_records.cu).
    sbf::DevBuf rb_dense, rb_norm, rb_meta, rb_hits, rb_stats;

    // Host threads that expand bit-packed query results into host bytes
    // (sbf_expand.cpp), created on first use; expand_threads < 0 until the
    // first host-output query decides (0 = download bytes).
    sbf::ExpandPool* expand = nullptr;
    int expand_threads = -1;

    uint64_t kmers_of(uint64_t symbols) const;
    // Windows of a byte sequence (symbols = bytes / width).
    uint64_t kmers_of_bytes(uint64_t bytes) const { return kmers_of(bytes / width); }
    // Dense packing: 64 / bits symbols per 64-bit word (32 for DNA).
    uint64_t dense_per_word() const { return 64u / gen.bits; }
    uint64_t dense_words(uint64_t symbols) const {
        return (symbols + dense_per_word() - 1) / dense_per_word();
    }
    // The ragged host pipeline and the server work on one-byte symbols only;
    // SBF_OK or an invalid-argument error.
    int require_byte_symbols(const char* what) const;
    int stage_record_batch(const char* h_seq, uint64_t len, const sbf_record_range* r, uint64_t n,
                           cudaStream_t st, std::vector<uint64_t>& out_off, uint64_t& norm_len);
    int record_pass(bool query, uint64_t n, uint64_t norm_len, uint8_t* d_hits, cudaStream_t st,
                    std::vector<uint64_t>& valid, std::vector<uint64_t>& positive,
                    uint64_t* total_valid);
    int launch(bool query, bool dense, const void* input, uint64_t input_bytes, uint64_t n_kmers,
               uint8_t* out, cudaStream_t st, uint32_t* out_bits = nullptr) const;
    int host_pipeline(bool query, bool dense, const void* h_in, uint64_t in_bytes,
                      uint64_t n_kmers, uint8_t* out_host, uint8_t* out_dev, cudaStream_t st,
                      uint32_t* bits_host = nullptr);
    int check_device_error(cudaStream_t st) const;
};

namespace sbf {
void ragged_release(sbf_filter* f);
void fastq_device_release(sbf_filter* f);
// The filter's pool for expanding bit-packed results into host bytes, or
// nullptr when host-output queries download bytes (sbf_expand.cpp).
ExpandPool* host_expand_pool(sbf_filter* f);
// Checks that records are ordered, non-overlapping and inside [0, len)
// (normalized_record_batch.hpp:123-147); large batches are checked on several
// host threads.  `total_bytes`, when given, receives the sum of the record
// lengths.
int validate_ranges(uint64_t len, const sbf_record_range* r, uint64_t n,
                    uint64_t* total_bytes = nullptr);
// Host record batches without the symbol-alignment check of the public entry
// points (FASTX chunks hold records of any length; normalisation pads each
// to a symbol boundary).
int insert_record_batch_impl(sbf_filter* f, const char* h_seq, uint64_t len,
                             const sbf_record_range* ranges, uint64_t n, sbf_stream_t stream,
                             sbf_insert_report* report);
int query_record_batch_impl(sbf_filter* f, const char* h_seq, uint64_t len,
                            const sbf_record_range* ranges, uint64_t n, sbf_stream_t stream,
                            sbf_query_report* report, sbf_record_query_cb consume, void* user);
}  // namespace sbf
