/*
 * sbf_b200.h -- C ABI of the B200 Super Bloom engine (libsbf_b200.so).
 *
 * Each entry point replaces one member of the reference's header-only
 * `cusbf::filter<Config>` class (include/cusbf/filter.cuh of tdortman/cuSBF);
 * the reference line each one stands in for is cited beside it.  Arguments
 * are plain pointers and sizes; streams are `cudaStream_t` values passed as
 * `sbf_stream_t` (NULL = legacy default stream).  Pointers documented as
 * "device" must be device-accessible; "host" pointers may be pageable.
 *
 * Every function returns an `sbf_status` (0 = success).  The non-zero codes
 * are the reference's error categories (include/cusbf/error.hpp:67-73) plus
 * one; `sbf_last_error_message()` returns the calling thread's message for
 * the last failure.  The C++ headers in include/cusbf/ translate them into
 * `cusbf::Result<T>`.
 *
 * Functions ending in `_async` do not synchronise the stream (as in the
 * reference); the others synchronise before returning.  A filter object is
 * not thread safe: callers serialise calls per filter, as with the
 * reference (filter.cuh:840 shares mutable staging across const methods).
 */
#ifndef SBF_B200_H
#define SBF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* sbf_stream_t;
typedef struct sbf_filter sbf_filter_t;

typedef enum {
    SBF_OK = 0,
    SBF_ERR_CUDA = 1,             /* ErrorCategory::cuda             */
    SBF_ERR_IO = 2,               /* ErrorCategory::io               */
    SBF_ERR_FASTX_PARSE = 3,      /* ErrorCategory::fastx_parse      */
    SBF_ERR_INVALID_ARGUMENT = 4, /* ErrorCategory::invalid_argument */
    SBF_ERR_RESOURCE = 5,         /* ErrorCategory::resource         */
} sbf_status;

/* Alphabet ids (include/cusbf/Alphabet.cuh:113-220).  The GPU engine
 * implements the DNA alphabet; the others are rejected with
 * SBF_ERR_INVALID_ARGUMENT by sbf_filter_create. */
enum { SBF_ALPHABET_DNA = 0, SBF_ALPHABET_DNA_TRIPLET = 1, SBF_ALPHABET_PROTEIN = 2 };

/* Record range inside a dense batch (include/cusbf/Fastx.hpp:24-29). */
typedef struct {
    uint64_t sequence_offset;
    uint64_t sequence_bytes;
} sbf_record_range;

/* FastxInsertReport (include/cusbf/Fastx.hpp:151-158). */
typedef struct {
    uint64_t records_indexed;
    uint64_t indexed_bases;
    uint64_t inserted_kmers;
} sbf_insert_report;

/* FastxQueryReport (include/cusbf/Fastx.hpp:161-170). */
typedef struct {
    uint64_t records_queried;
    uint64_t queried_bases;
    uint64_t queried_kmers;
    uint64_t positive_kmers;
} sbf_query_report;

/* ---- errors --------------------------------------------------------- */

/* Message of the calling thread's last failure ("" if none). */
const char* sbf_last_error_message(void);
/* cudaError_t of the calling thread's last SBF_ERR_CUDA failure. */
int sbf_last_cuda_error(void);
/* Library version string. */
const char* sbf_version(void);

/* ---- construction (filter.cuh:108-130) ------------------------------- */

/* Creates a filter for Config<k, s, m, hashes, 256, alphabet> with at least
 * `requested_bits` bits: the shard count is bit_ceil(max(1,
 * ceil(requested_bits / 256))), and the words are cleared (filter.cuh:108-120).
 * Configurations not compiled into the library return
 * SBF_ERR_INVALID_ARGUMENT. */
int sbf_filter_create(uint32_t k, uint32_t s, uint32_t m, uint32_t hashes, int alphabet,
                      uint64_t requested_bits, sbf_filter_t** out);
/* Releases device storage and staging buffers (filter.cuh:130). */
void sbf_filter_destroy(sbf_filter_t* filter);

/* Zeroes every word and synchronises `stream` (filter.cuh:793-803). */
int sbf_filter_clear(sbf_filter_t* filter, sbf_stream_t stream);
/* Allocated capacity in bits (filter.cuh:826-828). */
uint64_t sbf_filter_bits(const sbf_filter_t* filter);
/* Number of 256-bit shards (filter.cuh:831-833). */
uint64_t sbf_filter_num_shards(const sbf_filter_t* filter);
/* Device pointer to the shard words: num_shards * 4 little-endian uint64
 * words, shard i at words [4i, 4i+4) (filter.cuh:137-142, filter_ref). */
int sbf_filter_words(const sbf_filter_t* filter, uint64_t** d_words, uint64_t* n_words);
/* Fraction of set bits, synchronous (filter.cuh:810-823). */
int sbf_filter_load_factor(sbf_filter_t* filter, sbf_stream_t stream, double* out);
/* Windows of a byte sequence of `bytes` bytes (symbols - k + 1, or 0). */
uint64_t sbf_filter_kmer_count(const sbf_filter_t* filter, uint64_t bytes);

/* ---- byte sequences -------------------------------------------------- */

/* insert_sequence_async (filter.cuh:179-190): device bytes; `kmers_out`
 * receives the window count (0 if shorter than k). */
int sbf_insert_sequence_async(sbf_filter_t* filter, const char* d_seq, uint64_t bytes,
                              sbf_stream_t stream, uint64_t* kmers_out);
/* insert_sequence (filter.cuh:154-167): host bytes, staged through pinned
 * memory in chunks that overlap copies with kernels; synchronises. */
int sbf_insert_sequence(sbf_filter_t* filter, const char* h_seq, uint64_t bytes,
                        sbf_stream_t stream, uint64_t* kmers_out);
/* contains_sequence_async (filter.cuh:464-474): one byte per window written
 * to device `d_out` (capacity `out_len`); windows with an invalid symbol
 * read 0.  Sequences shorter than k leave `d_out` untouched. */
int sbf_contains_sequence_async(const sbf_filter_t* filter, const char* d_seq, uint64_t bytes,
                                uint8_t* d_out, uint64_t out_len, sbf_stream_t stream);
/* contains_sequence(string_view, device_span) (filter.cuh:486-501). */
int sbf_contains_sequence_to_device(const sbf_filter_t* filter, const char* h_seq,
                                    uint64_t bytes, uint8_t* d_out, uint64_t out_len,
                                    sbf_stream_t stream);
/* contains_sequence(string_view) (filter.cuh:514-533): host in, host out. */
int sbf_contains_sequence(const sbf_filter_t* filter, const char* h_seq, uint64_t bytes,
                          uint8_t* h_out, uint64_t out_len, sbf_stream_t stream);

/* ---- dense 2-bit input (filter.cuh:207-322, dense_packed.hpp) -------- */

/* Words needed for `num_symbols` dense symbols (dense_packed.hpp:20-22). */
uint64_t sbf_dense_packed_word_count(uint64_t num_symbols);
/* pack_dense_sequence_device (dense_packed.hpp:58-74). */
int sbf_pack_dense_device(const char* d_seq, uint64_t num_symbols, uint64_t* d_words,
                          sbf_stream_t stream);
/* pack_dense_sequence (dense_packed.hpp:36-50), on the host. */
int sbf_pack_dense_host(const char* h_seq, uint64_t num_symbols, uint64_t* h_words);
int sbf_insert_dense_packed_async(sbf_filter_t* filter, const uint64_t* d_words,
                                  uint64_t n_words, uint64_t num_symbols, sbf_stream_t stream,
                                  uint64_t* kmers_out);
int sbf_insert_dense_packed(sbf_filter_t* filter, const uint64_t* h_words, uint64_t n_words,
                            uint64_t num_symbols, sbf_stream_t stream, uint64_t* kmers_out);
int sbf_contains_dense_packed_async(const sbf_filter_t* filter, const uint64_t* d_words,
                                    uint64_t n_words, uint64_t num_symbols, uint8_t* d_out,
                                    uint64_t out_len, sbf_stream_t stream);
int sbf_contains_dense_packed_to_device(const sbf_filter_t* filter, const uint64_t* h_words,
                                        uint64_t n_words, uint64_t num_symbols, uint8_t* d_out,
                                        uint64_t out_len, sbf_stream_t stream);
int sbf_contains_dense_packed(const sbf_filter_t* filter, const uint64_t* h_words,
                              uint64_t n_words, uint64_t num_symbols, uint8_t* h_out,
                              uint64_t out_len, sbf_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* SBF_B200_H */
