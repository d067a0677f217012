// sbf_records.cu -- record batches: separator injection, query layout, per-record
// counts, and the record-batch entry points of the C ABI.
//
// Semantics follow the reference (tdortman/cuSBF):
//   * normalisation: records are joined with one separator symbol ('N' for
//     DNA) between consecutive records once any content has been written;
//     trailing partial symbols pad with separators first
//     (include/cusbf/normalized_record_batch.hpp:113-121, :209-276);
//   * range validation (normalized_record_batch.hpp:123-147, filter.cuh:848-876);
//   * query layout: hit_offset = logical_offset / symbolWidth, hit_count =
//     symbols - k + 1, total = windows of the whole normalised sequence
//     (include/cusbf/detail/query_layout.cuh:42-72);
//   * per-record valid k-mers (normalized_record_batch.hpp:88-110) and
//     positive k-mers (include/cusbf/detail/count_positive_kmers.cuh:21-45).
// The reference normalises on the host with memcpy; here the dense record
// bytes are copied to the device once and a gather kernel injects the
// separators, and per-record counts come from one segmented device pass.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/sbf_b200.h"
#include "sbf_host.h"
#include "sbf_internal.h"

using namespace sbf;

namespace sbf {

// Separator byte between normalised records (Alphabet::separator: '*' for
// proteins, 'N' for DNA and DNA triplets).
uint8_t separator_of(int alphabet) { return alphabet == SBF_ALPHABET_PROTEIN ? '*' : 'N'; }

// Whether the symbol at p encodes as valid (Alphabet::encode != invalidSymbol).
bool symbol_valid(int alphabet, const char* p) {
    auto dna = [](char c) {
        const uint8_t u = static_cast<uint8_t>(c) & 0xDFu;
        return u == 'A' || u == 'C' || u == 'G' || u == 'T';
    };
    if (alphabet == SBF_ALPHABET_PROTEIN)
        return static_cast<uint8_t>((static_cast<uint8_t>(p[0]) & 0xDFu) - 'A') < 26;
    if (alphabet == SBF_ALPHABET_DNA_TRIPLET) return dna(p[0]) && dna(p[1]) && dna(p[2]);
    return dna(p[0]);
}

// ---------------------------------------------------------------------------
// Host layout
// ---------------------------------------------------------------------------

// Checks records [lo, hi), the first against the end of record lo - 1.
// Returns 0, 1 (out of order or overlapping) or 2 (outside the sequence) for
// the first bad record, and the segment's byte total.
static int check_range_segment(uint64_t len, const sbf_record_range* r, uint64_t lo, uint64_t hi,
                               uint64_t* total) {
    uint64_t next = lo ? r[lo - 1].sequence_offset + r[lo - 1].sequence_bytes : 0;
    uint64_t sum = 0;
    for (uint64_t i = lo; i < hi; ++i) {
        if (r[i].sequence_offset < next) return 1;
        if (r[i].sequence_offset > len || r[i].sequence_bytes > len - r[i].sequence_offset)
            return 2;
        next = r[i].sequence_offset + r[i].sequence_bytes;
        sum += r[i].sequence_bytes;
    }
    *total = sum;
    return 0;
}

int validate_ranges(uint64_t len, const sbf_record_range* r, uint64_t n, uint64_t* total_bytes) {
    // One pass at about 1.5 ns per record: batches of tens of millions of
    // short reads are split over host threads so the check does not hold up
    // the uploads that follow it.
    constexpr uint64_t kPerThread = uint64_t{1} << 21;
    const uint64_t hw = std::max(1u, std::thread::hardware_concurrency());
    const uint64_t parts = std::max<uint64_t>(
        1, std::min<uint64_t>({(n + kPerThread - 1) / kPerThread, hw, 16}));
    std::vector<int> status(parts, 0);
    std::vector<uint64_t> sums(parts, 0);
    auto seg = [&](uint64_t p) {
        status[p] = check_range_segment(len, r, n * p / parts, n * (p + 1) / parts, &sums[p]);
    };
    if (parts == 1) {
        seg(0);
    } else {
        std::vector<std::thread> pool;
        pool.reserve(parts - 1);
        uint64_t started = 1;
        try {
            for (; started < parts; ++started) pool.emplace_back(seg, started);
        } catch (...) {
            // Fewer host threads than asked for: check the rest here.
        }
        for (uint64_t p = started; p < parts; ++p) seg(p);
        seg(0);
        for (auto& t : pool) t.join();
    }
    // The first bad record decides the message, as a serial scan would.
    for (uint64_t p = 0; p < parts; ++p) {
        if (status[p] == 1)
            return set_error(SBF_ERR_INVALID_ARGUMENT,
                             "record batch ranges must be ordered and non-overlapping");
        if (status[p] == 2)
            return set_error(SBF_ERR_INVALID_ARGUMENT,
                             "record batch range exceeds the source sequence");
    }
    if (total_bytes) {
        uint64_t t = 0;
        for (uint64_t s : sums) t += s;
        *total_bytes = t;
    }
    return SBF_OK;
}

// Record batches of multi-byte symbols must start and end on symbol
// boundaries (filter.cuh:865-873, normalized_record_batch.hpp:137-145).
int validate_alignment(uint32_t width, const sbf_record_range* r, uint64_t n) {
    if (width <= 1) return SBF_OK;
    for (uint64_t i = 0; i < n; ++i)
        if (r[i].sequence_offset % width != 0 || r[i].sequence_bytes % width != 0)
            return set_error(SBF_ERR_INVALID_ARGUMENT,
                             "record batch ranges must align to the configured alphabet symbol "
                             "width");
    return SBF_OK;
}

// Normalised offsets (write_record_boundary, normalized_record_batch.hpp:
// 209-232): before every record that follows non-empty content, the length
// is padded to a symbol boundary and one separator symbol (`width` bytes) is
// added.  Returns the normalised length.
uint64_t normalized_offsets(const sbf_record_range* r, uint64_t n, uint64_t* out_off,
                            uint32_t width) {
    uint64_t pos = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (pos != 0) pos += (width - pos % width) % width + width;
        out_off[i] = pos;
        pos += r[i].sequence_bytes;
    }
    return pos;
}

// ---------------------------------------------------------------------------
// Device kernels
// ---------------------------------------------------------------------------

// Normalised batch = record contents at their normalised offsets and the
// separator symbol everywhere else.  Each CTA builds segments of
// kGatherSegment output bytes (grid-strided): it fills the segment with
// separators, then copies the parts of the records that overlap it, so a
// single huge record is spread over the whole grid and many small ones share
// a CTA.
constexpr uint64_t kGatherSegment = 1u << 16;

__global__ void normalize_gather_kernel(const uint8_t* dense, uint64_t dense_base,
                                        const sbf_record_range* ranges, const uint64_t* out_off,
                                        uint64_t n, uint8_t* out, uint64_t norm_len,
                                        uint8_t separator) {
    __shared__ uint64_t first;
    for (uint64_t seg = blockIdx.x; seg * kGatherSegment < norm_len; seg += gridDim.x) {
        const uint64_t s0 = seg * kGatherSegment;
        const uint64_t s1 = s0 + kGatherSegment < norm_len ? s0 + kGatherSegment : norm_len;
        for (uint64_t x = s0 + threadIdx.x; x < s1; x += blockDim.x) out[x] = separator;
        if (threadIdx.x == 0) {
            // First record whose normalised end is past the segment start.
            uint64_t lo = 0, hi = n;
            while (lo < hi) {
                const uint64_t mid = (lo + hi) >> 1;
                if (out_off[mid] + ranges[mid].sequence_bytes > s0)
                    hi = mid;
                else
                    lo = mid + 1;
            }
            first = lo;
        }
        __syncthreads();
        for (uint64_t r = first; r < n && out_off[r] < s1; ++r) {
            const uint64_t beg = out_off[r];
            const uint64_t end = beg + ranges[r].sequence_bytes;
            const uint64_t a = beg > s0 ? beg : s0;
            const uint64_t b = end < s1 ? end : s1;
            const uint8_t* src = dense + (ranges[r].sequence_offset - dense_base) + (a - beg);
            for (uint64_t x = threadIdx.x; a + x < b; x += blockDim.x) out[a + x] = src[x];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Device staging of a host record batch
// ---------------------------------------------------------------------------

// Grow-only device buffer owned by a filter.
int DevBuf::ensure(size_t bytes) {
    if (bytes <= cap) return SBF_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    const size_t want = std::max<size_t>(bytes, 4096);
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(SBF_ERR_RESOURCE, "cannot allocate %zu bytes of device staging", want);
    }
    cap = want;
    return SBF_OK;
}

void DevBuf::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
}

}  // namespace sbf

#define SBF_CUDA(expr)                                      \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) return cuda_fail(_e, #expr); \
    } while (0)
#define SBF_TRY(expr)                \
    do {                             \
        int _s = (expr);             \
        if (_s != SBF_OK) return _s; \
    } while (0)

static inline cudaStream_t S(sbf_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// Stages a host record batch on the device: dense bytes + ranges + offsets,
// gathers the normalised sequence.  Fills `layout` (host) and returns the
// normalised length in `norm_len`.
int sbf_filter::stage_record_batch(const char* h_seq, uint64_t len, const sbf_record_range* r,
                                   uint64_t n, cudaStream_t st, std::vector<uint64_t>& out_off,
                                   uint64_t& norm_len) {
    SBF_TRY(validate_ranges(len, r, n));
    out_off.resize(n);
    norm_len = normalized_offsets(r, n, out_off.data(), width);
    if (n == 0 || norm_len == 0) return SBF_OK;
    // The dense span covering every record.
    uint64_t lo = r[0].sequence_offset, hi = 0;
    for (uint64_t i = 0; i < n; ++i) hi = std::max(hi, r[i].sequence_offset + r[i].sequence_bytes);
    const uint64_t span = hi - lo;
    SBF_TRY(rb_dense.ensure(span + 16));
    SBF_TRY(rb_norm.ensure(norm_len + 16));
    SBF_TRY(rb_meta.ensure(n * (2 * sizeof(sbf_record_range) + sizeof(uint64_t)) + 64));
    auto* d_ranges = static_cast<sbf_record_range*>(rb_meta.ptr);
    auto* d_off = reinterpret_cast<uint64_t*>(d_ranges + n);
    // The records' places in the normalised buffer: the ranges of the
    // ragged pass that inserts or queries it.
    std::vector<sbf_record_range> norm(n);
    for (uint64_t i = 0; i < n; ++i) norm[i] = sbf_record_range{out_off[i], r[i].sequence_bytes};
    SBF_CUDA(cudaMemcpyAsync(rb_dense.ptr, h_seq + lo, span, cudaMemcpyHostToDevice, st));
    SBF_CUDA(cudaMemcpyAsync(d_ranges, r, n * sizeof(sbf_record_range), cudaMemcpyHostToDevice, st));
    SBF_CUDA(cudaMemcpyAsync(d_off, out_off.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    SBF_CUDA(cudaMemcpyAsync(d_off + n, norm.data(), n * sizeof(sbf_record_range),
                             cudaMemcpyHostToDevice, st));
    const uint64_t segs = (norm_len + kGatherSegment - 1) / kGatherSegment;
    const uint64_t ctas = std::min<uint64_t>(segs, static_cast<uint64_t>(sms) * 8);
    normalize_gather_kernel<<<static_cast<unsigned>(ctas), 256, 0, st>>>(
        static_cast<const uint8_t*>(rb_dense.ptr), lo, d_ranges, d_off, n,
        static_cast<uint8_t*>(rb_norm.ptr), norm_len, separator_of(alphabet));
    SBF_CUDA(cudaGetLastError());
    // The host layout vector must stay alive until the copies complete.
    SBF_CUDA(cudaStreamSynchronize(st));
    return SBF_OK;
}

// One ragged pass over the staged normalised batch: inserts or queries it
// and returns per-record valid (and, for queries, positive) windows, counted
// in the kernel's epilogue.  d_hits (query, optional) receives the hit bytes
// in the normalised layout.
int sbf_filter::record_pass(bool query, uint64_t n, uint64_t norm_len, uint8_t* d_hits,
                            cudaStream_t st, std::vector<uint64_t>& valid,
                            std::vector<uint64_t>& positive, uint64_t* total_valid) {
    valid.assign(n, 0);
    positive.assign(n, 0);
    *total_valid = 0;
    const uint64_t windows = kmers_of_bytes(norm_len);
    if (n == 0 || windows == 0) return SBF_OK;
    SBF_TRY(rb_stats.ensure((2 * n + 2) * sizeof(uint64_t) + 64));
    auto* d_counts = static_cast<uint64_t*>(rb_stats.ptr);
    auto* d_valid = d_counts + 2;
    auto* d_pos = d_valid + n;
    const auto* d_norm = reinterpret_cast<const sbf_record_range*>(
        reinterpret_cast<const uint64_t*>(static_cast<const sbf_record_range*>(rb_meta.ptr) + n) + n);
    const char* seq = static_cast<const char*>(rb_norm.ptr);
    SBF_CUDA(cudaMemsetAsync(d_counts, 0, 2 * sizeof(uint64_t), st));
    unsigned long long tot[2] = {0, 0};
    if (query) {
        SBF_TRY(sbf_ragged_contains_counts_async(this, seq, norm_len, d_norm, n, d_hits, windows,
                                                 d_valid, d_pos, d_counts,
                                                 reinterpret_cast<sbf_stream_t>(st)));
        SBF_CUDA(cudaMemcpyAsync(valid.data(), d_valid, n * 8, cudaMemcpyDeviceToHost, st));
        SBF_CUDA(cudaMemcpyAsync(positive.data(), d_pos, n * 8, cudaMemcpyDeviceToHost, st));
    } else {
        SBF_TRY(sbf_ragged_insert_async(this, seq, norm_len, d_norm, n, d_counts,
                                        reinterpret_cast<sbf_stream_t>(st)));
    }
    SBF_CUDA(cudaMemcpyAsync(tot, d_counts, sizeof(tot), cudaMemcpyDeviceToHost, st));
    SBF_CUDA(cudaStreamSynchronize(st));
    *total_valid = tot[0];
    return SBF_OK;
}

// ---------------------------------------------------------------------------
// C ABI: host helpers (no GPU)
// ---------------------------------------------------------------------------

extern "C" int sbf_validate_record_batch(uint64_t len, const sbf_record_range* ranges,
                                         uint64_t n) {
    if (n && !ranges) return set_error(SBF_ERR_INVALID_ARGUMENT, "ranges pointer is null");
    return validate_ranges(len, ranges, n);
}

extern "C" int sbf_validate_record_batch_for(int alphabet, uint64_t len,
                                             const sbf_record_range* ranges, uint64_t n) {
    uint32_t bits = 0, width = 0;
    if (!alphabet_geometry(alphabet, &bits, &width))
        return set_error(SBF_ERR_INVALID_ARGUMENT, "unknown alphabet %d", alphabet);
    if (n && !ranges) return set_error(SBF_ERR_INVALID_ARGUMENT, "ranges pointer is null");
    SBF_TRY(validate_ranges(len, ranges, n));
    return validate_alignment(width, ranges, n);
}

// estimate_normalized_batch_bytes (normalized_record_batch.hpp:185-200).
extern "C" uint64_t sbf_normalized_batch_bytes_for(int alphabet, const sbf_record_range* ranges,
                                                   uint64_t n) {
    uint32_t bits = 0, width = 0;
    if (!alphabet_geometry(alphabet, &bits, &width)) return 0;
    uint64_t size = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (i != 0 || size != 0) size += (width - size % width) % width + width;
        size += ranges[i].sequence_bytes;
    }
    return size;
}

extern "C" uint64_t sbf_normalized_batch_bytes(const sbf_record_range* ranges, uint64_t n) {
    return sbf_normalized_batch_bytes_for(SBF_ALPHABET_DNA, ranges, n);
}

// normalize_record_batch (normalized_record_batch.hpp:235-276) for any
// alphabet: records at their normalised offsets, separator symbols between
// them, and each record's valid windows (valid_record_kmer_count, :88-110).
extern "C" int sbf_normalize_record_batch_for(int alphabet, uint32_t k, const char* h_seq,
                                              uint64_t len, const sbf_record_range* ranges,
                                              uint64_t n, char* out, uint64_t out_cap,
                                              uint64_t* out_len,
                                              sbf_normalized_record* records_out) {
    uint32_t bits = 0, width = 0;
    if (!alphabet_geometry(alphabet, &bits, &width))
        return set_error(SBF_ERR_INVALID_ARGUMENT, "unknown alphabet %d", alphabet);
    if (n && (!ranges || !h_seq)) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    SBF_TRY(validate_ranges(len, ranges, n));
    SBF_TRY(validate_alignment(width, ranges, n));
    std::vector<uint64_t> off(n);
    const uint64_t total = normalized_offsets(ranges, n, off.data(), width);
    if (out_len) *out_len = total;
    if (out && out_cap < total)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "normalised output buffer is too small");
    const char sep = static_cast<char>(separator_of(alphabet));
    uint64_t written = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const char* src = h_seq + ranges[i].sequence_offset;
        const uint64_t size = ranges[i].sequence_bytes;
        if (out) {
            std::memset(out + written, sep, off[i] - written);
            std::memcpy(out + off[i], src, size);
            written = off[i] + size;
        }
        if (records_out) {
            const uint64_t syms = size / width;
            uint64_t valid = 0;
            if (syms >= k) {
                uint64_t invalid = 0;
                auto bad = [&](uint64_t t) { return !symbol_valid(alphabet, src + t * width); };
                for (uint64_t t = 0; t < k; ++t) invalid += bad(t);
                valid = invalid == 0;
                for (uint64_t t = 1; t + k <= syms; ++t) {
                    invalid -= bad(t - 1);
                    invalid += bad(t + k - 1);
                    valid += invalid == 0;
                }
            }
            records_out[i] = sbf_normalized_record{i, ranges[i].sequence_offset, size, valid};
        }
    }
    return SBF_OK;
}

extern "C" int sbf_normalize_record_batch(uint32_t k, const char* h_seq, uint64_t len,
                                          const sbf_record_range* ranges, uint64_t n, char* out,
                                          uint64_t out_cap, uint64_t* out_len,
                                          sbf_normalized_record* records_out) {
    return sbf_normalize_record_batch_for(SBF_ALPHABET_DNA, k, h_seq, len, ranges, n, out, out_cap,
                                          out_len, records_out);
}

// QueryLayout::build (detail/query_layout.cuh:42-72): hit offsets are
// normalised symbol positions.
extern "C" int sbf_query_layout_for(int alphabet, uint32_t k,
                                    const sbf_normalized_record* records, uint64_t n,
                                    sbf_query_layout_record* out, uint64_t* total_hits) {
    uint32_t bits = 0, width = 0;
    if (!alphabet_geometry(alphabet, &bits, &width))
        return set_error(SBF_ERR_INVALID_ARGUMENT, "unknown alphabet %d", alphabet);
    if (n && (!records || !out)) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    auto kmers = [&](uint64_t bytes) { return bytes / width < k ? 0 : bytes / width - k + 1; };
    uint64_t logical = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (logical != 0) logical += (width - logical % width) % width + width;
        const uint64_t size = records[i].size;
        out[i] = sbf_query_layout_record{records[i].record_index, records[i].input_offset, size,
                                         records[i].valid_kmers, logical / width, kmers(size)};
        logical += size;
    }
    if (total_hits) *total_hits = kmers(logical);
    return SBF_OK;
}

extern "C" int sbf_query_layout(uint32_t k, const sbf_normalized_record* records, uint64_t n,
                                sbf_query_layout_record* out, uint64_t* total_hits) {
    return sbf_query_layout_for(SBF_ALPHABET_DNA, k, records, n, out, total_hits);
}

// ---------------------------------------------------------------------------
// C ABI: device record batches (separators already in place)
// ---------------------------------------------------------------------------

extern "C" int sbf_insert_record_batch_async(sbf_filter_t* f, const char* d_seq, uint64_t len,
                                             const sbf_record_range* ranges, uint64_t n,
                                             sbf_stream_t stream, uint64_t* kmers_out) {
    if (kmers_out) *kmers_out = 0;
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    if (n && !ranges) return set_error(SBF_ERR_INVALID_ARGUMENT, "ranges pointer is null");
    SBF_TRY(validate_ranges(len, ranges, n));
    SBF_TRY(validate_alignment(f->width, ranges, n));
    uint64_t total = 0;
    for (uint64_t i = 0; i < n; ++i) total += f->kmers_of_bytes(ranges[i].sequence_bytes);
    if (kmers_out) *kmers_out = total;
    if (total == 0) return SBF_OK;
    return f->launch(false, false, d_seq, len, f->kmers_of_bytes(len), nullptr, S(stream));
}

extern "C" int sbf_contains_record_batch_async(const sbf_filter_t* f, const char* d_seq,
                                               uint64_t len, const sbf_record_range* ranges,
                                               uint64_t n, uint8_t* d_out, uint64_t out_len,
                                               sbf_stream_t stream) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    if (n && !ranges) return set_error(SBF_ERR_INVALID_ARGUMENT, "ranges pointer is null");
    SBF_TRY(validate_ranges(len, ranges, n));
    SBF_TRY(validate_alignment(f->width, ranges, n));
    const uint64_t total = f->kmers_of_bytes(len);
    if (total == 0) return SBF_OK;
    if (!d_out || out_len < total)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "record batch query output span is too small");
    return f->launch(true, false, d_seq, len, total, d_out, S(stream));
}

// ---------------------------------------------------------------------------
// C ABI: host record batches
// ---------------------------------------------------------------------------

int sbf::insert_record_batch_impl(sbf_filter* f, const char* h_seq, uint64_t len,
                                  const sbf_record_range* ranges, uint64_t n, sbf_stream_t stream,
                                  sbf_insert_report* report) {
    if (n && (!ranges || !h_seq)) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    cudaStream_t st = S(stream);
    std::vector<uint64_t> off;
    uint64_t norm_len = 0;
    SBF_TRY(f->stage_record_batch(h_seq, len, ranges, n, st, off, norm_len));
    sbf_insert_report rep{n, 0, 0};
    for (uint64_t i = 0; i < n; ++i) rep.indexed_bases += ranges[i].sequence_bytes;
    if (f->kmers_of_bytes(norm_len)) {
        std::vector<uint64_t> valid, pos;
        SBF_TRY(f->record_pass(false, n, norm_len, nullptr, st, valid, pos, &rep.inserted_kmers));
        SBF_TRY(f->check_device_error(st));
    }
    if (report) *report = rep;
    return SBF_OK;
}

int sbf::query_record_batch_impl(sbf_filter* f, const char* h_seq, uint64_t len,
                                 const sbf_record_range* ranges, uint64_t n, sbf_stream_t stream,
                                 sbf_query_report* report, sbf_record_query_cb consume,
                                 void* user) {
    if (n && (!ranges || !h_seq)) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    cudaStream_t st = S(stream);
    std::vector<uint64_t> off;
    uint64_t norm_len = 0;
    SBF_TRY(f->stage_record_batch(h_seq, len, ranges, n, st, off, norm_len));
    sbf_query_report rep{n, 0, 0, 0};
    for (uint64_t i = 0; i < n; ++i) rep.queried_bases += ranges[i].sequence_bytes;
    const uint64_t windows = f->kmers_of_bytes(norm_len);
    std::vector<uint64_t> valid(n, 0), pos(n, 0);
    std::vector<uint8_t> hits;
    if (windows) {
        // Hit bytes are written only when a consumer reads them.
        uint8_t* d_hits = nullptr;
        if (consume) {
            SBF_TRY(f->rb_hits.ensure(windows + 64));
            d_hits = static_cast<uint8_t*>(f->rb_hits.ptr);
        }
        uint64_t total = 0;
        SBF_TRY(f->record_pass(true, n, norm_len, d_hits, st, valid, pos, &total));
        if (consume) {
            hits.resize(windows);
            SBF_CUDA(cudaMemcpyAsync(hits.data(), d_hits, windows, cudaMemcpyDeviceToHost, st));
            SBF_CUDA(cudaStreamSynchronize(st));
        }
        SBF_TRY(f->check_device_error(st));
    }
    for (uint64_t i = 0; i < n; ++i) {
        rep.queried_kmers += valid[i];
        rep.positive_kmers += pos[i];
    }
    if (consume) {
        for (uint64_t i = 0; i < n; ++i) {
            const uint64_t size = ranges[i].sequence_bytes;
            const uint64_t hc = f->kmers_of_bytes(size);
            sbf_record_view v{i,
                              h_seq + ranges[i].sequence_offset,
                              size,
                              size,
                              valid[i],
                              pos[i],
                              hc ? hits.data() + off[i] / f->width : nullptr,
                              hc};
            if (consume(user, &v) != 0)
                return set_error(SBF_ERR_ABORTED, "record consumer aborted the query");
        }
    }
    if (report) *report = rep;
    return SBF_OK;
}

extern "C" int sbf_insert_record_batch(sbf_filter_t* f, const char* h_seq, uint64_t len,
                                       const sbf_record_range* ranges, uint64_t n,
                                       sbf_stream_t stream, sbf_insert_report* report) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    if (n && !ranges) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    SBF_TRY(validate_alignment(f->width, ranges, n));
    return insert_record_batch_impl(f, h_seq, len, ranges, n, stream, report);
}

extern "C" int sbf_query_record_batch(const sbf_filter_t* cf, const char* h_seq, uint64_t len,
                                      const sbf_record_range* ranges, uint64_t n,
                                      sbf_stream_t stream, sbf_query_report* report,
                                      sbf_record_query_cb consume, void* user) {
    auto* f = const_cast<sbf_filter*>(cf);
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    if (n && !ranges) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    SBF_TRY(validate_alignment(f->width, ranges, n));
    return query_record_batch_impl(f, h_seq, len, ranges, n, stream, report, consume, user);
}
