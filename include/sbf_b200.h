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
    SBF_ERR_ABORTED = 6,          /* a consumer callback asked to stop */
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

/* NormalizedRecord (include/cusbf/normalized_record_batch.hpp:20-29). */
typedef struct {
    uint64_t record_index;
    uint64_t input_offset;
    uint64_t size;
    uint64_t valid_kmers;
} sbf_normalized_record;

/* QueryLayoutRecord (include/cusbf/detail/query_layout.cuh:13-20). */
typedef struct {
    uint64_t record_index;
    uint64_t input_offset;
    uint64_t size;
    uint64_t valid_kmers;
    uint64_t hit_offset;
    uint64_t hit_count;
} sbf_query_layout_record;

/* RecordQueryView (include/cusbf/Fastx.hpp:135-148): one record's result,
 * valid only during the callback.  `hits` has `n_hits` bytes (1 = present). */
typedef struct {
    uint64_t record_index;
    const char* sequence;
    uint64_t sequence_bytes;
    uint64_t queried_bases;
    uint64_t queried_kmers;
    uint64_t positive_kmers;
    const uint8_t* hits;
    uint64_t n_hits;
} sbf_record_view;

/* Per-record consumer of the record-batch query API (RecordQueryConsumer,
 * Fastx.hpp:223-226).  Returning non-zero aborts the call, which then
 * returns SBF_ERR_ABORTED (the C++ headers rethrow the consumer's exception,
 * as the reference lets it propagate); the filter stays usable. */
typedef int (*sbf_record_query_cb)(void* user, const sbf_record_view* record);

/* FastxRecordView (include/cusbf/Fastx.hpp:173-188). */
typedef struct {
    uint64_t record_index;
    const char* header;
    uint64_t header_bytes;
    const char* sequence;
    uint64_t sequence_bytes;
    uint64_t queried_bases;
    uint64_t queried_kmers;
    uint64_t positive_kmers;
    const uint8_t* hits;
    uint64_t n_hits;
} sbf_fastx_record_view;

/* Per-record consumer of the FASTX query APIs (FastxRecordConsumer,
 * Fastx.hpp:235-238); non-zero aborts like sbf_record_query_cb. */
typedef int (*sbf_fastx_record_cb)(void* user, const sbf_fastx_record_view* record);

/* Pull-style input for the FASTX stream APIs: copies up to `cap` bytes into
 * `buf` and returns the count, 0 at end of input, or -1 on a read error. */
typedef int64_t (*sbf_read_fn)(void* user, char* buf, uint64_t cap);

/* ---- errors --------------------------------------------------------- */

/* Message of the calling thread's last failure ("" if none). */
const char* sbf_last_error_message(void);
/* Source location of the calling thread's last SBF_ERR_FASTX_PARSE failure
 * (FastxParseError::location, error.hpp:53-56): file, 1-based line, column. */
int sbf_last_error_location(const char** file, uint32_t* line, uint32_t* column);
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
/* Which kernels a filter runs (no reference counterpart; the reference
 * compiles every Config into the caller): 0 = tile kernels compiled into the
 * library, 1 = the same tile kernels compiled at run time for this
 * configuration (NVRTC, cached under $SBF_JIT_CACHE, off with SBF_JIT=0),
 * 2 = runtime-parameterised kernels (other alphabets, or when run-time
 * compilation is off or fails).  All three give identical results. */
int sbf_filter_kernel_path(const sbf_filter_t* filter);
/* Device pointer to the shard words: num_shards * 4 little-endian uint64
 * words, shard i at words [4i, 4i+4) (filter.cuh:137-142, filter_ref). */
int sbf_filter_words(const sbf_filter_t* filter, uint64_t** d_words, uint64_t* n_words);
/* Fraction of set bits, synchronous (filter.cuh:810-823). */
int sbf_filter_load_factor(sbf_filter_t* filter, sbf_stream_t stream, double* out);
/* Windows of a byte sequence of `bytes` bytes (symbols - k + 1, or 0). */
uint64_t sbf_filter_kmer_count(const sbf_filter_t* filter, uint64_t bytes);

/* ---- bit-packed query results (no reference counterpart) ----------------
 * The same answers as sbf_contains_sequence*, one bit per window: bit i % 32
 * of word i / 32 is window i's hit (bits past the last window are 0), an 8x
 * smaller result to store or copy back.  n_words >= ceil(windows / 32). */
int sbf_contains_sequence_bits_async(const sbf_filter_t* filter, const char* d_seq,
                                     uint64_t bytes, uint32_t* d_bits, uint64_t n_words,
                                     sbf_stream_t stream);
/* Host input and host bit output through the pinned chunk pipeline. */
int sbf_contains_sequence_bits(const sbf_filter_t* filter, const char* h_seq, uint64_t bytes,
                               uint32_t* h_bits, uint64_t n_words, sbf_stream_t stream);
/* Host only, no GPU work: expands bit-packed results into one byte per
 * window (out[i] = bit i % 32 of bits[i / 32], 0 or 1) on up to `threads`
 * host threads (0 = half the hardware threads, at most 4).  The host-output
 * queries (sbf_contains_sequence, sbf_ragged_query, ...) download bits and
 * expand them this way on hosts with at least 8 hardware threads, with 4
 * threads (SBF_HOST_EXPAND_THREADS overrides); SBF_HOST_EXPAND=0 makes them
 * download bytes instead, =1 always expand. */
int sbf_expand_result_bits(const uint32_t* bits, uint64_t n_windows, uint8_t* out,
                           uint32_t threads);
/* Host threads that host-output queries of filters created from now on will
 * expand bit-packed results with (0: they download one byte per window). */
int sbf_host_expand_threads(void);

/* ---- persistence (no reference counterpart) ------------------------------
 * A saved filter is a 40-byte header (magic "SBFB200", version, k, s, m,
 * hashes, alphabet, shard count) followed by the shard words in the
 * reference's filter_block layout.  Synchronous on `stream`. */
int sbf_filter_save(const sbf_filter_t* filter, const char* path, sbf_stream_t stream);
/* Configuration and size of a saved filter (to create a matching filter). */
int sbf_filter_file_info(const char* path, uint32_t* k, uint32_t* s, uint32_t* m,
                         uint32_t* hashes, uint64_t* filter_bits);
/* Replaces the filter's words with a saved filter of the same configuration
 * and shard count; on any error the filter is left unchanged
 * (SBF_ERR_IO: unreadable or malformed file; SBF_ERR_INVALID_ARGUMENT:
 * another configuration or size). */
int sbf_filter_load(sbf_filter_t* filter, const char* path, sbf_stream_t stream);

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
/* The same three for any alphabet (SBF_ALPHABET_*): 64 / bits symbols per
 * word (32 DNA, 12 protein, 10 DNA triplets); num_symbols symbols of
 * symbolWidth input bytes each (3 for DNA triplets). */
uint64_t sbf_dense_packed_word_count_for(int alphabet, uint64_t num_symbols);
int sbf_pack_dense_host_for(int alphabet, const char* h_seq, uint64_t num_symbols,
                            uint64_t* h_words);
int sbf_pack_dense_device_for(int alphabet, const char* d_seq, uint64_t num_symbols,
                              uint64_t* d_words, sbf_stream_t stream);
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
/* Dense input with bit-packed results (no reference counterpart): bit i % 32
 * of word i / 32 is window i's result; with 2-bit input this moves a quarter
 * byte in and an eighth of a byte out per window.  d_bits 4-byte aligned. */
int sbf_contains_dense_packed_bits_async(const sbf_filter_t* filter, const uint64_t* d_words,
                                         uint64_t n_words, uint64_t num_symbols, uint32_t* d_bits,
                                         uint64_t n_bit_words, sbf_stream_t stream);
int sbf_contains_dense_packed_bits(const sbf_filter_t* filter, const uint64_t* h_words,
                                   uint64_t n_words, uint64_t num_symbols, uint32_t* h_bits,
                                   uint64_t n_bit_words, sbf_stream_t stream);

/* ---- record batches (filter.cuh:338-400, :549-622) ----------------- */

/* validateRecordBatch (normalized_record_batch.hpp:123-147): ranges must be
 * ordered, non-overlapping and inside `len` bytes.  Host only. */
int sbf_validate_record_batch(uint64_t len, const sbf_record_range* ranges, uint64_t n);
/* estimate_normalized_batch_bytes (normalized_record_batch.hpp:179-194). */
uint64_t sbf_normalized_batch_bytes(const sbf_record_range* ranges, uint64_t n);
/* normalize_record_batch_into (normalized_record_batch.hpp:289-304), on the
 * host: joins records with one 'N' and fills per-record metadata
 * (`records_out` may be NULL; `out` may be NULL to size the output). */
int sbf_normalize_record_batch(uint32_t k, const char* h_seq, uint64_t len,
                               const sbf_record_range* ranges, uint64_t n, char* out,
                               uint64_t out_cap, uint64_t* out_len,
                               sbf_normalized_record* records_out);
/* QueryLayout::build (include/cusbf/detail/query_layout.cuh:42-72). */
int sbf_query_layout(uint32_t k, const sbf_normalized_record* records, uint64_t n,
                     sbf_query_layout_record* out, uint64_t* total_hits);
/* The four above for any alphabet (SBF_ALPHABET_*): the DNA-triplet alphabet
 * needs record ranges aligned to its 3-byte symbols; records are joined by
 * one separator symbol (symbolWidth bytes of 'N', or '*' for proteins) after
 * padding to a symbol boundary, valid windows are counted over symbols, and
 * hit offsets are normalised symbol positions. */
int sbf_validate_record_batch_for(int alphabet, uint64_t len, const sbf_record_range* ranges,
                                  uint64_t n);
uint64_t sbf_normalized_batch_bytes_for(int alphabet, const sbf_record_range* ranges, uint64_t n);
int sbf_normalize_record_batch_for(int alphabet, uint32_t k, const char* h_seq, uint64_t len,
                                   const sbf_record_range* ranges, uint64_t n, char* out,
                                   uint64_t out_cap, uint64_t* out_len,
                                   sbf_normalized_record* records_out);
int sbf_query_layout_for(int alphabet, uint32_t k, const sbf_normalized_record* records,
                         uint64_t n, sbf_query_layout_record* out, uint64_t* total_hits);

/* insert_record_batch (filter.cuh:338-364): host records, separators injected
 * on the device; synchronises. */
int sbf_insert_record_batch(sbf_filter_t* filter, const char* h_seq, uint64_t len,
                            const sbf_record_range* ranges, uint64_t n, sbf_stream_t stream,
                            sbf_insert_report* report);
/* insert_record_batch_async (filter.cuh:385-400): device sequence with the
 * separators already in place; `kmers_out` = attempted windows per record. */
int sbf_insert_record_batch_async(sbf_filter_t* filter, const char* d_seq, uint64_t len,
                                  const sbf_record_range* ranges, uint64_t n,
                                  sbf_stream_t stream, uint64_t* kmers_out);
/* query_record_batch (filter.cuh:549-582): aggregate report, and with a
 * non-NULL `consume` one callback per record in order. */
int sbf_query_record_batch(const sbf_filter_t* filter, const char* h_seq, uint64_t len,
                           const sbf_record_range* ranges, uint64_t n, sbf_stream_t stream,
                           sbf_query_report* report, sbf_record_query_cb consume, void* user);
/* contains_record_batch_async (filter.cuh:603-622). */
int sbf_contains_record_batch_async(const sbf_filter_t* filter, const char* d_seq, uint64_t len,
                                    const sbf_record_range* ranges, uint64_t n, uint8_t* d_out,
                                    uint64_t out_len, sbf_stream_t stream);

/* Per-record counts of a device record batch (separators already in place,
 * as for sbf_contains_record_batch_async) without allocating anything: no
 * reference counterpart.  valid_out[i] = valid k-mer windows of record i
 * (valid_record_kmer_count, normalized_record_batch.hpp:88-110) and, with a
 * non-NULL d_hits (the batch's output of sbf_contains_record_batch_async,
 * hits_len bytes), positive_out[i] = its set hits
 * (count_positive_kmers_per_record, detail/count_positive_kmers.cuh:21-45);
 * positive_out[i] = 0 without d_hits.  Both outputs are host arrays of n.
 *
 * For callers that may not allocate device memory at call time: a serving
 * loop whose device memory is reserved once at start-up and must not grow
 * while requests are in flight, or an allocator hook that must not re-enter
 * the CUDA allocator it belongs to.  The other record-batch entry points may
 * grow device buffers inside the filter; this one only uses an 8 MiB scratch
 * area compiled into the library (held by every device that loads the
 * library until the process exits), and calls no cudaMalloc or cudaFree.
 * Limit: n <= 262144 records; larger batches return
 * SBF_ERR_INVALID_ARGUMENT.  The filter's device must be the current device
 * (else SBF_ERR_INVALID_ARGUMENT).  The first call on a device looks the
 * scratch address up (cudaGetSymbolAddress), so make that first call before
 * any stream capture.  Calls share the scratch, which keeps the last call's
 * contents: calls on one device must not overlap on the GPU (serialise them
 * on one stream or host thread), or they race.  The call is synchronous: it
 * copies `ranges` from host memory, copies the counts back to the host
 * arrays, and returns after the stream has reached the end of the call. */
int sbf_record_batch_counts_noalloc(const sbf_filter_t* filter, const char* d_seq, uint64_t len,
                                    const sbf_record_range* ranges, uint64_t n,
                                    const uint8_t* d_hits, uint64_t hits_len,
                                    sbf_stream_t stream, uint64_t* valid_out,
                                    uint64_t* positive_out);

/* ---- Ragged batches (no reference counterpart) ------------------------
 *
 * Many records of uneven length in one buffer, processed in place by one
 * persistent kernel launch whose CTAs take tiles from a device work queue.
 * Records are (offset, bytes) ranges into the buffer, sorted by offset and
 * non-overlapping (gaps allowed).  Exactly the windows that lie inside one
 * record are inserted / queried: the result equals one insert_sequence /
 * contains_sequence per record (filter.cuh:154-190, :464-533), the
 * reference's "plain per-record launch".
 *
 * Query output layout: one byte per window of the whole buffer, the window
 * starting at byte p at out[p]; record r's hits are
 * out[offset_r, offset_r + bytes_r - k + 1).  Windows that cross a record
 * boundary or touch a byte outside every record read 0.  Output length is
 * len - k + 1 (0 when len < k). */

/* Host pipeline knobs; zero fields take defaults. */
typedef struct {
    uint64_t chunk_bytes; /* bytes staged per chunk (default 64 MiB insert, 256 MiB
                             query; min 4096) */
    uint32_t stages;      /* chunks in flight, 1..4 (default 2 insert, 3 query) */
    uint32_t ctas_per_sm; /* resident CTAs per SM, 0 = occupancy limit */
    uint32_t use_graph;   /* replay each chunk's device work as a CUDA graph */
} sbf_ragged_tuning;

/* Device-resident ragged insert: d_seq (len bytes) and d_ranges (n records)
 * on the device; ranges are trusted (unsorted ranges give unspecified
 * results, never out-of-bounds access).  With d_counts non-NULL (device,
 * 2 x uint64, zeroed by the caller) valid windows are added to d_counts[0].
 * Asynchronous on `stream`. */
int sbf_ragged_insert_async(sbf_filter_t* filter, const char* d_seq, uint64_t len,
                            const sbf_record_range* d_ranges, uint64_t n, uint64_t* d_counts,
                            sbf_stream_t stream);
/* Device-resident ragged query into d_out (out_len >= len - k + 1); valid
 * windows are added to d_counts[0] and positive ones to d_counts[1]. */
int sbf_ragged_contains_async(const sbf_filter_t* filter, const char* d_seq, uint64_t len,
                              const sbf_record_range* d_ranges, uint64_t n, uint8_t* d_out,
                              uint64_t out_len, uint64_t* d_counts, sbf_stream_t stream);
/* The device-resident ragged query with per-record counts computed in the
 * query kernel's epilogue (the reference computes them in a second pass:
 * count_positive_kmers_per_record, detail/count_positive_kmers.cuh:21-45,
 * called from filter.cuh:1055).  d_record_valid[r] and d_record_positive[r]
 * (device, n x uint64, zeroed here) receive record r's valid and positive
 * windows.  d_out is optional: NULL computes the counts without writing any
 * hit bytes; otherwise it is filled as by sbf_ragged_contains_async. */
int sbf_ragged_contains_counts_async(const sbf_filter_t* filter, const char* d_seq, uint64_t len,
                                     const sbf_record_range* d_ranges, uint64_t n,
                                     uint8_t* d_out, uint64_t out_len, uint64_t* d_record_valid,
                                     uint64_t* d_record_positive, uint64_t* d_counts,
                                     sbf_stream_t stream);
/* Host batches through the chunked pipeline (ranges validated as for
 * record batches).  `tuning` NULL uses the tuning table entry for the
 * batch's shape when there is one, else defaults.  Synchronous. */
int sbf_ragged_insert(sbf_filter_t* filter, const char* h_seq, uint64_t len,
                      const sbf_record_range* ranges, uint64_t n,
                      const sbf_ragged_tuning* tuning, sbf_stream_t stream,
                      sbf_insert_report* report);
int sbf_ragged_query(const sbf_filter_t* filter, const char* h_seq, uint64_t len,
                     const sbf_record_range* ranges, uint64_t n, uint8_t* h_out,
                     uint64_t out_len, const sbf_ragged_tuning* tuning, sbf_stream_t stream,
                     sbf_query_report* report);
/* sbf_ragged_query with bit-packed results (window i of the buffer -> bit
 * i % 32 of h_bits[i / 32]; n_words >= ceil((len - k + 1) / 32)): an eighth
 * of the download.  Chunks hold a multiple of 32 windows. */
int sbf_ragged_query_bits(const sbf_filter_t* filter, const char* h_seq, uint64_t len,
                          const sbf_record_range* ranges, uint64_t n, uint32_t* h_bits,
                          uint64_t n_words, const sbf_ragged_tuning* tuning, sbf_stream_t stream,
                          sbf_query_report* report);
/* Times chunk size x stages x graph replay, then CTAs per SM for the
 * winner, on a prefix of the batch
 * (sample_bytes, 0 = 1 GiB), stores the fastest in the tuning table
 * (SBF_TUNE_TABLE, default $HOME/.cache/cusbf_b200/ragged_tuning.tsv) under
 * the batch's shape (operation, configuration, log2 bytes, log2 mean record
 * bytes) and returns it.  An insert tune inserts the prefix. */
int sbf_ragged_autotune(sbf_filter_t* filter, int query, const char* h_seq, uint64_t len,
                        const sbf_record_range* ranges, uint64_t n, uint64_t sample_bytes,
                        sbf_stream_t stream, sbf_ragged_tuning* chosen);
/* Tuning table entry for a shape; SBF_ERR_INVALID_ARGUMENT (defaults in
 * *out) when the table has none. */
int sbf_ragged_tuning_lookup(const sbf_filter_t* filter, int query, uint64_t len, uint64_t n,
                             sbf_ragged_tuning* out);

/* ---- Sharded multi-rank insert (no reference counterpart) --------------
 *
 * Replaces, when W ranks (one per GPU) split one input, the single-GPU insert
 * (insert_sequence_kmers_kernel, detail/kernels.cuh:214-242, which ORs each
 * super-k-mer run's word masks into its shard, filter_ref.cuh:94-108):
 *   1. each rank emits the run records of its windows (sbf_emit_runs_async);
 *   2. the caller routes every record to the rank owning its shard (shards
 *      split into W contiguous ranges; cusbf_b200/sharded.py does this with
 *      one torch.distributed all-to-all);
 *   3. each rank ORs the records it owns into its shard range
 *      (sbf_apply_runs_async), and an all-gather of the ranges gives every
 *      rank the filter one GPU would build from the whole input.
 * DNA configurations compiled into the library only. */

/* Run records of the windows of device bytes d_seq[0, len): record i is
 * d_shards[i] and the four word masks d_masks[4i, 4i+4) (16-byte aligned).
 * d_count (device, 2 x uint64) receives the records emitted and the valid
 * windows; records beyond `capacity` are counted but not stored, so a count
 * above capacity means the call must be repeated with larger buffers. */
int sbf_emit_runs_async(const sbf_filter_t* filter, const char* d_seq, uint64_t len,
                        uint32_t* d_shards, uint64_t* d_masks, uint64_t capacity,
                        uint64_t* d_count, sbf_stream_t stream);
/* ORs n device records into the filter; every shard must lie in
 * [shard_lo, shard_hi), else the device error word is set and the next
 * sbf_filter_synchronize returns SBF_ERR_CUDA. */
int sbf_apply_runs_async(sbf_filter_t* filter, const uint32_t* d_shards, const uint64_t* d_masks,
                         uint64_t n, uint64_t shard_lo, uint64_t shard_hi, sbf_stream_t stream);
/* Waits for `stream` and reports a device-side error of the filter's kernels
 * (a staging wait that ran out, a misrouted run record) as SBF_ERR_CUDA. */
int sbf_filter_synchronize(const sbf_filter_t* filter, sbf_stream_t stream);

/* ---- Request server (no reference counterpart) ------------------------
 *
 * Keeps a filter resident and serves insert and query requests from any
 * number of host threads with continuous batching: a worker thread forms
 * each batch from the longest run of queued requests of one operation (in
 * arrival order) that fits max_batch_bytes, admits it when the device
 * staging ring (staging_bytes, the memory budget) has room and fewer than
 * max_inflight batches are on the GPU, and runs it as one ragged pass with
 * uploads, kernels and downloads on separate streams.  Kernels run in
 * arrival order, so every result equals one-request-at-a-time execution.
 * While a server runs, its filter must not be used directly. */
typedef struct sbf_server sbf_server_t;

typedef struct {
    uint64_t staging_bytes;      /* device staging budget (default 16 GiB) */
    uint64_t max_batch_bytes;    /* sequence bytes per batch (default 256 MiB) */
    uint64_t pinned_bytes;       /* pinned host staging (default 1 GiB) */
    uint32_t max_inflight;       /* batches on the GPU at once (default 16) */
    uint32_t max_batch_requests; /* 0 = unlimited; 1 = one request per launch */
    uint32_t use_graph;          /* replay each batch's kernels as a CUDA graph */
} sbf_server_config;

typedef struct {
    int status;        /* SBF_OK or the failure */
    double latency_s;  /* completion - arrival */
    uint64_t windows;  /* k-mer windows of the request's span */
    double arrival_s;  /* sbf_server_now() clock */
    double done_s;
} sbf_server_request_info;

typedef struct {
    uint64_t requests, batches, query_windows, insert_windows;
    double wall_s; /* first arrival to last completion */
    double p50_s, p99_s, p999_s, max_s, mean_s;
    double mean_batch_requests;
    double worker_busy_s;    /* worker time spent staging and launching batches */
    double admission_wait_s; /* worker time waiting for staging-ring space */
    double slot_wait_s;      /* worker time waiting for a free in-flight slot with work queued */
} sbf_server_stats;

/* config NULL = defaults.  Allocates the staging ring and starts the worker
 * and completion threads. */
int sbf_server_create(sbf_filter_t* filter, const sbf_server_config* config,
                      sbf_server_t** out);
/* Finishes queued work, then stops the threads and frees the server. */
void sbf_server_destroy(sbf_server_t* server);
/* The server's clock (seconds, monotonic) for arrival stamps. */
double sbf_server_now(void);
/* Queues a request: op 0 = insert, 1 = query, 2 = query with bit-packed
 * results (out[] as 32-bit words, bit i % 32 of word i / 32 for window i;
 * out_len >= 4 * ceil((span - k + 1) / 32)), 3 = query returning only
 * per-record counts (out[] as 2n uint64: record r's valid windows at 2r,
 * positive windows at 2r + 1; out_len >= 16 n).  op | 0x10: `base` holds
 * 2-bit dense-packed DNA words (sbf_pack_dense_host layout) and the ranges
 * count symbols; the words are unpacked on the GPU.  Records are (offset, bytes)
 * ranges into `base`, ordered and non-overlapping; the request's span is
 * [ranges[0].offset, end of ranges[n-1]).  A query writes one byte per
 * window of the span to out[0 .. span - k] (out_len >= span - k + 1): the
 * hit of the window starting at base + ranges[0].offset + i is out[i], and
 * windows not inside one record read 0.  base, ranges and out must stay
 * valid until the request completes; pinned buffers are copied directly.
 * arrival <= 0 stamps the request with sbf_server_now().  Returns a ticket. */
int sbf_server_submit(sbf_server_t* server, int op, const char* base,
                      const sbf_record_range* ranges, uint64_t n, uint8_t* out, uint64_t out_len,
                      double arrival, uint64_t* ticket);
/* Waits for a request (timeout_s <= 0: no limit) and forgets its ticket. */
int sbf_server_wait(sbf_server_t* server, uint64_t ticket, double timeout_s,
                    sbf_server_request_info* info);
/* Waits until every queued request has completed. */
int sbf_server_drain(sbf_server_t* server);
/* Latency percentiles and throughput counters since the last reset. */
int sbf_server_get_stats(sbf_server_t* server, int reset, sbf_server_stats* out);

/* ---- FASTA / FASTQ (filter.cuh:402-786, Fastx.hpp:297-481) ----------- */

/* Record consumer of sbf_fastx_scan: header (without '>'/'@') and sequence
 * of record `index`; non-zero stops the scan. */
typedef int (*sbf_fastx_scan_cb)(void* user, uint64_t index, const char* header,
                                 uint64_t header_bytes, const char* sequence,
                                 uint64_t sequence_bytes);
/* FastxReader::nextRecord (Fastx.hpp:314-354) over a whole input, host only:
 * one callback per record; parse errors as SBF_ERR_FASTX_PARSE. */
int sbf_fastx_scan(sbf_read_fn read, void* read_user, const char* source_name,
                   sbf_fastx_scan_cb consume, void* user, uint64_t* records_out);
/* The same over a plain or gzip file (openFastxFile, Fastx.hpp:470-481). */
int sbf_fastx_scan_file(const char* path, sbf_fastx_scan_cb consume, void* user,
                        uint64_t* records_out);

/* insert_fastx (filter.cuh:416-421): FASTA or FASTQ (format from the first
 * header; wrapped lines and CRLF accepted; FASTQ quality lengths checked)
 * read through `read`; records are accumulated into chunks whose device
 * staging stays within fill_fraction * (free memory - 64 MiB) (a fraction of
 * 0 or less flushes every record) and inserted as record batches, so no
 * k-mer spans two records.  `source_name` labels parse errors. */
int sbf_insert_fastx(sbf_filter_t* filter, sbf_read_fn read, void* read_user,
                     const char* source_name, double fill_fraction, sbf_stream_t stream,
                     sbf_insert_report* report);
/* insert_fastx_file (filter.cuh:437-452): plain or gzip-compressed file. */
int sbf_insert_fastx_file(sbf_filter_t* filter, const char* path, double fill_fraction,
                          sbf_stream_t stream, sbf_insert_report* report);
/* query_fastx / query_fastx_records (filter.cuh:632-735): aggregate report;
 * with a non-NULL `consume`, one FastxRecordView per record in source order. */
int sbf_query_fastx(const sbf_filter_t* filter, sbf_read_fn read, void* read_user,
                    const char* source_name, double fill_fraction, sbf_stream_t stream,
                    sbf_query_report* report, sbf_fastx_record_cb consume, void* user);
/* query_fastx_file / query_fastx_file_records (filter.cuh:654-735). */
int sbf_query_fastx_file(const sbf_filter_t* filter, const char* path, double fill_fraction,
                         sbf_stream_t stream, sbf_query_report* report,
                         sbf_fastx_record_cb consume, void* user);

#ifdef __cplusplus
}
#endif

#endif /* SBF_B200_H */
