// sbf_fastq_gpu.cu -- FASTQ and FASTA parsing on the GPU for the FASTX
// insert/query entry points.  The reference parses on the host (FastxReader,
// include/cusbf/Fastx.hpp:297-462, detail/fastx_buffer_reader.hpp:90-169);
// here a block of raw FASTQ text is uploaded as it is and
//
//   1. every newline is located (per-tile counts, one exclusive scan, then
//      each tile writes the positions of its newlines in order);
//   2. each record's four lines are checked in parallel (header starting
//      with '@', a sequence line that does not start with '+', a '+' line,
//      a quality line of the sequence's length; '\r' before '\n' ignored);
//   3. the sequence lines become the records of a ragged pass over the raw
//      text (records in place, no copy), so headers, '+' lines, qualities
//      and newlines are bytes outside every record.
//
// FASTA blocks use the same newline scan; each line's sequence bytes (none
// for '>' headers) are scanned into offsets and copied into one compacted
// buffer, header lines delimit records, and the block's last record is kept
// for the next block unless the input ends.
//
// Blocks whose structure is anything else (wrapped lines, blank lines,
// malformed records) are reported as irregular and the caller parses the
// rest of the input on the host with the reference's rules, so results and
// error locations are the reference's in every case.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstring>

#include "../../include/sbf_b200.h"
#include "sbf_fastq_gpu.h"
#include "sbf_host.h"
#include "sbf_internal.h"
#include "sbf_ragged.h"

namespace sbf {

namespace {

constexpr int kScanThreads = 256;

// A count that is either the host's `n` or, in a block replayed as a CUDA
// graph, read on the device from `dn` and clamped to the buffer capacity.
__device__ __forceinline__ uint64_t dev_count(uint64_t n, const unsigned long long* dn,
                                              uint64_t cap) {
    if (!dn) return n;
    const uint64_t v = *dn;
    return v < cap ? v : cap;
}
constexpr uint64_t kTileBytes = uint64_t{kScanThreads} * 256;  // 256 bytes per thread

__device__ __forceinline__ uint32_t newlines_in(const uint8_t* t, uint64_t a, uint64_t b) {
    uint32_t c = 0;
    uint64_t x = a;
    // 16-byte words where aligned (tiles and thread slices start aligned).
    for (; x + 16 <= b; x += 16) {
        const uint4 v = *reinterpret_cast<const uint4*>(t + x);
        c += __popc(__vcmpeq4(v.x, 0x0A0A0A0Au)) + __popc(__vcmpeq4(v.y, 0x0A0A0A0Au)) +
             __popc(__vcmpeq4(v.z, 0x0A0A0A0Au)) + __popc(__vcmpeq4(v.w, 0x0A0A0A0Au));
    }
    uint32_t bytes = c / 8;
    for (; x < b; ++x) bytes += t[x] == '\n';
    return bytes;
}

// Exclusive scan of the block's per-thread values (shared memory, 256 threads).
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* sh,
                                                         uint32_t* total) {
    const int tid = threadIdx.x;
    sh[tid] = v;
    __syncthreads();
    for (int o = 1; o < kScanThreads; o <<= 1) {
        const uint32_t add = tid >= o ? sh[tid - o] : 0u;
        __syncthreads();
        sh[tid] += add;
        __syncthreads();
    }
    const uint32_t incl = sh[tid];
    *total = sh[kScanThreads - 1];
    __syncthreads();
    return incl - v;
}

__global__ void tile_newlines_kernel(const uint8_t* t, uint64_t n, uint64_t* tile_count) {
    __shared__ uint32_t sh[kScanThreads];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kTileBytes;
    const uint64_t a = base + static_cast<uint64_t>(threadIdx.x) * 256;
    const uint64_t b = a + 256 < n ? a + 256 : n;
    const uint32_t c = a < n ? newlines_in(t, a, b) : 0u;
    uint32_t total;
    (void)block_exclusive_scan(c, sh, &total);
    if (threadIdx.x == 0) tile_count[blockIdx.x] = total;
}

// In-place exclusive scan of up to a few hundred thousand counts (one CTA).
__global__ void scan_counts_kernel(uint64_t* v, uint64_t n, uint64_t* total,
                                   const unsigned long long* dn = nullptr, uint64_t cap = 0) {
    __shared__ uint64_t part[1024];
    n = dev_count(n, dn, cap);
    const uint64_t per = (n + 1023) / 1024;
    const uint64_t a = threadIdx.x * per;
    const uint64_t b = a + per < n ? a + per : n;
    uint64_t s = 0;
    for (uint64_t i = a; i < b; ++i) s += v[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const uint64_t add = threadIdx.x >= static_cast<unsigned>(o) ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += add;
        __syncthreads();
    }
    uint64_t run = part[threadIdx.x] - s;
    for (uint64_t i = a; i < b; ++i) {
        const uint64_t x = v[i];
        v[i] = run;
        run += x;
    }
    if (threadIdx.x == 1023) *total = part[1023];
}

enum : unsigned int { kIrregular = 1u, kLineOverflow = 2u };
static_assert(kIrregular == kBlockIrregular && kLineOverflow == kBlockLineOverflow,
              "device flags are the block summary's");

// Newline positions in order; positions at or beyond `cap` are not stored
// and set kLineOverflow (the caller grows line_end and repeats the block).
__global__ void newline_positions_kernel(const uint8_t* t, uint64_t n, const uint64_t* tile_off,
                                         uint64_t* line_end, uint64_t cap, unsigned int* flags) {
    __shared__ uint32_t sh[kScanThreads];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kTileBytes;
    const uint64_t a = base + static_cast<uint64_t>(threadIdx.x) * 256;
    const uint64_t b = a + 256 < n ? a + 256 : n;
    const uint32_t c = a < n ? newlines_in(t, a, b) : 0u;
    uint32_t total;
    const uint32_t before = block_exclusive_scan(c, sh, &total);
    uint64_t out = tile_off[blockIdx.x] + before;
    bool over = false;
    for (uint64_t x = a; x < b; ++x)
        if (t[x] == '\n') {
            if (out < cap)
                line_end[out] = x;
            else
                over = true;
            ++out;
        }
    if (over) atomicOr(flags, kLineOverflow);
}

// One thread per record: lines 4r .. 4r+3.
__global__ void fastq_records_kernel(const uint8_t* t, const uint64_t* line_end, uint64_t n_rec,
                                     DevRange* seq, DevRange* hdr, unsigned int* flags,
                                     unsigned long long* bases,
                                     const unsigned long long* dn_lines = nullptr,
                                     uint64_t cap = 0) {
    if (dn_lines) n_rec = dev_count(0, dn_lines, cap) / 4;
    unsigned long long local = 0;
    for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n_rec;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t l = 4 * r;
        const uint64_t h0 = l == 0 ? 0 : line_end[l - 1] + 1;
        uint64_t h1 = line_end[l];
        const uint64_t s0 = h1 + 1;
        uint64_t s1 = line_end[l + 1];
        const uint64_t p0 = s1 + 1;
        const uint64_t q0 = line_end[l + 2] + 1;
        uint64_t q1 = line_end[l + 3];
        if (h1 > h0 && t[h1 - 1] == '\r') --h1;
        if (s1 > s0 && t[s1 - 1] == '\r') --s1;
        if (q1 > q0 && t[q1 - 1] == '\r') --q1;
        const bool ok = h1 > h0 && t[h0] == '@' && (s1 == s0 || t[s0] != '+') &&
                        line_end[l + 2] > p0 - 1 && t[p0] == '+' && q1 - q0 == s1 - s0;
        if (!ok) atomicOr(flags, kIrregular);
        seq[r] = DevRange{s0, s1 - s0};
        hdr[r] = DevRange{h0 + 1, h1 - h0 - 1};
        local += s1 - s0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xFFFFFFFFu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(bases, local);
}

// Bounds of line i without its '\n' and a trailing '\r', and whether it is a
// FASTA header ('>' first).
__device__ __forceinline__ bool fasta_line(const uint8_t* t, const uint64_t* line_end, uint64_t i,
                                           uint64_t* a_out, uint64_t* b_out) {
    const uint64_t a = i == 0 ? 0 : line_end[i - 1] + 1;
    uint64_t b = line_end[i];
    if (b > a && t[b - 1] == '\r') --b;
    *a_out = a;
    *b_out = b;
    return b > a && t[a] == '>';
}

// FASTA, one thread per line: sequence bytes of the line (0 for headers and
// '\r') and a header flag ('>' at the line start).
__global__ void fasta_lines_kernel(const uint8_t* t, const uint64_t* line_end, uint64_t n,
                                   uint64_t* len, uint64_t* hdr,
                                   const unsigned long long* dn = nullptr, uint64_t cap = 0) {
    n = dev_count(n, dn, cap);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t a, b;
        const bool h = fasta_line(t, line_end, i, &a, &b);
        hdr[i] = h ? 1 : 0;
        len[i] = h ? 0 : b - a;
    }
}

// One warp per line: copies sequence lines to their compacted offsets
// (`off`: exclusive scan of the line lengths).
__global__ void fasta_compact_kernel(const uint8_t* t, const uint64_t* line_end, uint64_t n,
                                     const uint64_t* off, uint8_t* comp,
                                     const unsigned long long* dn = nullptr, uint64_t cap = 0) {
    n = dev_count(n, dn, cap);
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t warps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t i = warp; i < n; i += warps) {
        uint64_t a, b;
        if (fasta_line(t, line_end, i, &a, &b)) continue;
        for (uint64_t x = lane; a + x < b; x += 32) comp[off[i] + x] = t[a + x];
    }
}

// One thread per line: header line i starts record hdr_scan[i] (headers
// before it), whose sequence starts at off[i].  `last` receives the last
// record's header line start and sequence start.
__global__ void fasta_records_kernel(const uint8_t* t, const uint64_t* line_end, uint64_t n,
                                     const uint64_t* off, const uint64_t* hdr_scan,
                                     uint64_t n_rec, DevRange* seq, DevRange* hdr,
                                     unsigned long long* last,
                                     const unsigned long long* dn = nullptr, uint64_t cap = 0,
                                     const unsigned long long* dn_rec = nullptr) {
    n = dev_count(n, dn, cap);
    if (dn_rec) n_rec = *dn_rec;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t a, b;
        if (!fasta_line(t, line_end, i, &a, &b)) continue;
        const uint64_t r = hdr_scan[i];
        hdr[r] = DevRange{a + 1, b - a - 1};
        seq[r].offset = off[i];
        if (r + 1 == n_rec) {
            last[0] = a;
            last[1] = off[i];
            last[2] = i;
        }
    }
}

// Record lengths once every record start is known.
__global__ void fasta_lengths_kernel(DevRange* seq, uint64_t n_rec, uint64_t total_seq,
                                     const unsigned long long* dn_rec = nullptr,
                                     const unsigned long long* d_total = nullptr) {
    if (dn_rec) n_rec = *dn_rec;
    if (d_total) total_seq = *d_total;
    for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n_rec;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t end = r + 1 < n_rec ? seq[r + 1].offset : total_seq;
        seq[r].bytes = end - seq[r].offset;
    }
}

// Sizes of the ragged pass of a FASTQ block parsed on the device, and the
// block summary.  ctl: [0] newlines, [1] flags, [2] sequence bytes.  A block
// that is irregular, overflows line_end or holds no record gets n_tiles = 0.
__global__ void fastq_sizes_kernel(const uint64_t* line_end, const unsigned long long* ctl,
                                   uint64_t cap, int64_t phase, uint32_t k, DevSizes* sz,
                                   BlockSummary* sum) {
    const uint64_t n_lines = ctl[0];
    const uint64_t flags = (ctl[1] & 0xFFFFFFFFull) | (n_lines > cap ? kLineOverflow : 0u);
    const uint64_t n_rec = n_lines > cap ? 0 : n_lines / 4;
    const bool ok = flags == 0 && n_rec > 0;
    const uint64_t base_len = n_rec ? line_end[4 * n_rec - 1] + 1 : 0;
    const uint64_t n_kmers = ok && base_len >= k ? base_len - k + 1 : 0;
    sz->input_bytes = ok ? base_len : 0;
    sz->n_kmers = n_kmers;
    sz->n_tiles = n_kmers ? (n_kmers + static_cast<uint64_t>(phase) + kTileKmers - 1) / kTileKmers : 0;
    sz->n_ranges = ok ? n_rec : 0;
    sum->lines = n_lines;
    sum->flags = flags;
    sum->bases = ctl[2];
    sum->consumed = base_len;
    sum->records = n_rec;
    sum->lines_used = 4 * n_rec;
}

// The same for a FASTA block.  ctl: [0] newlines, [1] flags, [3] compacted
// sequence bytes, [4] headers (records), [5..7] the last header's line start,
// sequence start and line.  Without `eof` the last record waits for the next
// block; a block without a header is irregular.
__global__ void fasta_sizes_kernel(const unsigned long long* ctl, uint64_t cap, uint64_t len,
                                   int eof, int64_t phase, uint32_t k, DevSizes* sz,
                                   BlockSummary* sum) {
    const uint64_t n_lines = ctl[0];
    const bool over = n_lines > cap;
    const uint64_t n_rec = over ? 0 : ctl[4];
    const uint64_t flags = (ctl[1] & 0xFFFFFFFFull) | (over ? kLineOverflow : 0u) |
                           (!over && n_rec == 0 ? kIrregular : 0u);
    const uint64_t use = n_rec == 0 ? 0 : (eof ? n_rec : n_rec - 1);
    const uint64_t base_len = use == 0 ? 0 : (eof ? ctl[3] : ctl[6]);
    const bool ok = flags == 0 && use > 0;
    const uint64_t n_kmers = ok && base_len >= k ? base_len - k + 1 : 0;
    sz->input_bytes = ok ? base_len : 0;
    sz->n_kmers = n_kmers;
    sz->n_tiles = n_kmers ? (n_kmers + static_cast<uint64_t>(phase) + kTileKmers - 1) / kTileKmers : 0;
    sz->n_ranges = ok ? use : 0;
    sum->lines = n_lines;
    sum->flags = flags;
    sum->bases = base_len;
    sum->consumed = use == 0 ? 0 : (eof ? len : ctl[5]);
    sum->records = use;
    sum->lines_used = use == 0 ? 0 : (eof ? n_lines : ctl[7]);
}

template <class T>
int grow(DevBuf& b, uint64_t count) {
    return b.ensure(count * sizeof(T) + 64);
}

}  // namespace

int FastqDevice::scan_lines(sbf_filter* f, const uint8_t* h_text, uint64_t len, cudaStream_t st,
                            uint64_t* n_lines_out) {
    (void)f;
    *n_lines_out = 0;
    const uint64_t tiles = (len + kTileBytes - 1) / kTileBytes;
    if (tiles > (uint64_t{1} << 20))
        return set_error(SBF_ERR_INVALID_ARGUMENT, "FASTX block too large for the device parser");
    int s;
    if ((s = text.ensure(len + 64)) != SBF_OK) return s;
    if ((s = grow<uint64_t>(tile_off, tiles + 2)) != SBF_OK) return s;
    if ((s = ctl.ensure(128)) != SBF_OK) return s;
    auto* d_text = static_cast<uint8_t*>(text.ptr);
    auto* d_tiles = static_cast<uint64_t*>(tile_off.ptr);
    auto* d_ctl = static_cast<unsigned long long*>(ctl.ptr);
    cudaError_t e;
    if ((e = cudaMemcpyAsync(d_text, h_text, len, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyAsync(fastx block)");
    if ((e = cudaMemsetAsync(d_ctl, 0, 64, st)) != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    tile_newlines_kernel<<<static_cast<unsigned>(tiles), kScanThreads, 0, st>>>(d_text, len, d_tiles);
    scan_counts_kernel<<<1, 1024, 0, st>>>(d_tiles, tiles, reinterpret_cast<uint64_t*>(d_ctl));
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "newline scan");
    unsigned long long n_lines = 0;
    if ((e = cudaMemcpyAsync(&n_lines, d_ctl, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyAsync(lines)");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    if (n_lines == 0) return SBF_OK;
    if ((s = grow<uint64_t>(line_end, n_lines + 1)) != SBF_OK) return s;
    newline_positions_kernel<<<static_cast<unsigned>(tiles), kScanThreads, 0, st>>>(
        d_text, len, d_tiles, static_cast<uint64_t*>(line_end.ptr), n_lines + 1,
        reinterpret_cast<unsigned int*>(d_ctl + 1));
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "newline_positions_kernel");
    *n_lines_out = n_lines;
    return SBF_OK;
}

int FastqDevice::parse(sbf_filter* f, const uint8_t* h_text, uint64_t len, cudaStream_t st,
                       FastqBlock* out) {
    *out = FastqBlock{};
    if (len == 0) return SBF_OK;
    uint64_t n_lines = 0;
    int s = scan_lines(f, h_text, len, st, &n_lines);
    if (s != SBF_OK) return s;
    out->lines = n_lines;
    const uint64_t n_rec = n_lines / 4;
    out->records = n_rec;
    if (n_rec == 0) return SBF_OK;
    if ((s = grow<DevRange>(seq, n_rec)) != SBF_OK) return s;
    if ((s = grow<DevRange>(hdr, n_rec)) != SBF_OK) return s;
    auto* d_text = static_cast<uint8_t*>(text.ptr);
    auto* d_le = static_cast<uint64_t*>(line_end.ptr);
    auto* d_ctl = static_cast<unsigned long long*>(ctl.ptr);  // [1] flags, [2] bases
    cudaError_t e;
    const uint64_t threads = std::min<uint64_t>(n_rec, static_cast<uint64_t>(f->sms) * 2048);
    fastq_records_kernel<<<static_cast<unsigned>((threads + 255) / 256), 256, 0, st>>>(
        d_text, d_le, n_rec, static_cast<DevRange*>(seq.ptr), static_cast<DevRange*>(hdr.ptr),
        reinterpret_cast<unsigned int*>(d_ctl + 1), d_ctl + 2);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "fastq_records_kernel");
    unsigned long long h[3] = {0, 0, 0};
    uint64_t last_end = 0;
    if ((e = cudaMemcpyAsync(h, d_ctl, sizeof h, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyAsync(flags)");
    if ((e = cudaMemcpyAsync(&last_end, d_le + 4 * n_rec - 1, 8, cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
        return cuda_fail(e, "cudaMemcpyAsync(line end)");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    out->regular = (h[1] & kIrregular) == 0;
    out->bases = h[2];
    out->consumed = last_end + 1;
    out->d_text = d_text;
    out->d_base = d_text;
    out->base_len = out->consumed;
    out->d_seq = static_cast<const DevRange*>(seq.ptr);
    out->d_hdr = static_cast<const DevRange*>(hdr.ptr);
    return SBF_OK;
}

int FastqDevice::parse_fasta(sbf_filter* f, const uint8_t* h_text, uint64_t len, bool eof,
                             cudaStream_t st, FastqBlock* out) {
    *out = FastqBlock{};
    out->compacted = true;
    if (len == 0) return SBF_OK;
    uint64_t n_lines = 0;
    int s = scan_lines(f, h_text, len, st, &n_lines);
    if (s != SBF_OK) return s;
    out->lines = n_lines;
    if (n_lines == 0) return SBF_OK;
    if ((s = grow<uint64_t>(line_len, n_lines + 1)) != SBF_OK) return s;
    if ((s = grow<uint64_t>(line_hdr, n_lines + 1)) != SBF_OK) return s;
    auto* d_text = static_cast<uint8_t*>(text.ptr);
    auto* d_le = static_cast<uint64_t*>(line_end.ptr);
    auto* d_len = static_cast<uint64_t*>(line_len.ptr);
    auto* d_hdrf = static_cast<uint64_t*>(line_hdr.ptr);
    auto* d_ctl = static_cast<unsigned long long*>(ctl.ptr);  // [3] seq total, [4] headers, [5..7] last header
    cudaError_t e;
    const unsigned lblocks =
        static_cast<unsigned>(std::min<uint64_t>((n_lines + 255) / 256, static_cast<uint64_t>(f->sms) * 32));
    fasta_lines_kernel<<<lblocks, 256, 0, st>>>(d_text, d_le, n_lines, d_len, d_hdrf);
    scan_counts_kernel<<<1, 1024, 0, st>>>(d_len, n_lines, reinterpret_cast<uint64_t*>(d_ctl + 3));
    scan_counts_kernel<<<1, 1024, 0, st>>>(d_hdrf, n_lines, reinterpret_cast<uint64_t*>(d_ctl + 4));
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "fasta line scan");
    unsigned long long tot[2] = {0, 0};
    if ((e = cudaMemcpyAsync(tot, d_ctl + 3, 16, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyAsync(fasta totals)");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    const uint64_t total_seq = tot[0], n_rec = tot[1];
    if (n_rec == 0) {
        out->regular = false;  // no header among the complete lines
        return SBF_OK;
    }
    if ((s = comp.ensure(total_seq + 64)) != SBF_OK) return s;
    if ((s = grow<DevRange>(seq, n_rec)) != SBF_OK) return s;
    if ((s = grow<DevRange>(hdr, n_rec)) != SBF_OK) return s;
    auto* d_comp = static_cast<uint8_t*>(comp.ptr);
    const uint64_t warps = std::min<uint64_t>(n_lines, static_cast<uint64_t>(f->sms) * 64);
    fasta_compact_kernel<<<static_cast<unsigned>((warps * 32 + 255) / 256), 256, 0, st>>>(
        d_text, d_le, n_lines, d_len, d_comp);
    fasta_records_kernel<<<lblocks, 256, 0, st>>>(d_text, d_le, n_lines, d_len, d_hdrf, n_rec,
                                                  static_cast<DevRange*>(seq.ptr),
                                                  static_cast<DevRange*>(hdr.ptr), d_ctl + 5);
    fasta_lengths_kernel<<<static_cast<unsigned>(std::min<uint64_t>((n_rec + 255) / 256, 4096)),
                           256, 0, st>>>(static_cast<DevRange*>(seq.ptr), n_rec, total_seq);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "fasta records");
    unsigned long long last[3] = {0, 0, 0};  // last header: line start, sequence start, line
    if ((e = cudaMemcpyAsync(last, d_ctl + 5, 24, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyAsync(last header)");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    const uint64_t use = eof ? n_rec : n_rec - 1;
    out->records = use;
    out->lines = eof ? n_lines : last[2];  // lines of the records processed
    out->consumed = eof ? len : last[0];
    out->base_len = eof ? total_seq : last[1];
    out->bases = out->base_len;
    out->d_text = d_text;
    out->d_base = d_comp;
    out->d_seq = static_cast<const DevRange*>(seq.ptr);
    out->d_hdr = static_cast<const DevRange*>(hdr.ptr);
    return SBF_OK;
}

int FastqDevice::run(sbf_filter* f, bool query, const FastqBlock& b, cudaStream_t st,
                     bool want_views, uint64_t* valid, uint64_t* positive) {
    *valid = *positive = 0;
    if (b.records == 0) return SBF_OK;
    int s;
    if ((s = counts.ensure(64)) != SBF_OK) return s;
    auto* d_counts = static_cast<unsigned long long*>(counts.ptr);
    cudaError_t e;
    if ((e = cudaMemsetAsync(d_counts, 0, 16, st)) != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    // The records of this block end at b.base_len: the ragged pass covers
    // exactly those bytes of d_base (the text for FASTQ, the compacted
    // sequences for FASTA).
    const uint64_t len = b.base_len;
    const uint64_t windows = f->kmers_of(len);
    uint8_t* d_hits = nullptr;
    const bool views = query && want_views;
    unsigned long long *d_valid = nullptr, *d_pos = nullptr;
    if (views) {
        if ((s = rec_counts.ensure(b.records * 16 + 64)) != SBF_OK) return s;
        d_valid = static_cast<unsigned long long*>(rec_counts.ptr);
        d_pos = d_valid + b.records;
    }
    if (query) {
        if ((s = out.ensure(windows + 64)) != SBF_OK) return s;
        d_hits = static_cast<uint8_t*>(out.ptr);
        // With record views the per-record counts come from the query
        // kernel's epilogue.
        s = views ? sbf_ragged_contains_counts_async(
                        f, reinterpret_cast<const char*>(b.d_base), len,
                        reinterpret_cast<const sbf_record_range*>(b.d_seq), b.records, d_hits,
                        windows, reinterpret_cast<uint64_t*>(d_valid),
                        reinterpret_cast<uint64_t*>(d_pos), reinterpret_cast<uint64_t*>(d_counts),
                        reinterpret_cast<sbf_stream_t>(st))
                  : sbf_ragged_contains_async(f, reinterpret_cast<const char*>(b.d_base), len,
                                              reinterpret_cast<const sbf_record_range*>(b.d_seq),
                                              b.records, d_hits, windows,
                                              reinterpret_cast<uint64_t*>(d_counts),
                                              reinterpret_cast<sbf_stream_t>(st));
    } else {
        s = sbf_ragged_insert_async(f, reinterpret_cast<const char*>(b.d_base), len,
                                    reinterpret_cast<const sbf_record_range*>(b.d_seq), b.records,
                                    reinterpret_cast<uint64_t*>(d_counts),
                                    reinterpret_cast<sbf_stream_t>(st));
    }
    if (s != SBF_OK) return s;
    unsigned long long h[2] = {0, 0};
    if ((e = cudaMemcpyAsync(h, d_counts, 16, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyAsync(counts)");
    if (views) {
        // The record table, per-record counts and hits for the callbacks.
        if (b.compacted) {
            if ((s = h_comp.ensure(len + 64)) != SBF_OK) return s;
            if (len && (e = cudaMemcpyAsync(h_comp.p, b.d_base, len, cudaMemcpyDeviceToHost, st)) !=
                           cudaSuccess)
                return cuda_fail(e, "cudaMemcpyAsync(fasta sequences)");
        }
        h_seq.resize(b.records);
        h_hdr.resize(b.records);
        h_valid.resize(b.records);
        h_pos.resize(b.records);
        if ((s = h_hits.ensure(windows + 64)) != SBF_OK) return s;
        if ((e = cudaMemcpyAsync(h_seq.data(), b.d_seq, b.records * 16, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(h_hdr.data(), b.d_hdr, b.records * 16, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(h_valid.data(), d_valid, b.records * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(h_pos.data(), d_pos, b.records * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(h_hits.p, d_hits, windows, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return cuda_fail(e, "cudaMemcpyAsync(record views)");
    }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    if ((s = f->check_device_error(st)) != SBF_OK) return s;
    *valid = h[0];
    *positive = h[1];
    return SBF_OK;
}

bool FastqDevice::graph_usable(const sbf_filter* f) {
    // Graph kernel nodes take the kernels compiled into the library; the
    // generic kernels do not read device-side sizes.
    return f->ks && !f->ks->jit && f->ks != generic_kernels() && f->width == 1;
}

int FastqDevice::run_block_graph(sbf_filter* f, bool query, bool fasta, const uint8_t* h_text,
                                 uint64_t len, bool eof, cudaStream_t st, BlockSummary* out) {
    *out = BlockSummary{};
    if (len == 0) return SBF_OK;
    const int s = launch_block_graph(f, query, fasta, h_text, len, eof, st);
    return s != SBF_OK ? s : finish_block_graph(f, st, out);
}

int FastqDevice::finish_block_graph(sbf_filter* f, cudaStream_t st, BlockSummary* out) {
    cudaError_t e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    const int s = f->check_device_error(st);
    if (s != SBF_OK) return s;
    *out = *static_cast<const BlockSummary*>(h_summary.p);
    if (out->flags & kLineOverflow) line_cap = out->lines + 1;
    return SBF_OK;
}

int FastqDevice::launch_block_graph(sbf_filter* f, bool query, bool fasta, const uint8_t* h_text,
                                    uint64_t len, bool eof, cudaStream_t st) {
    const uint64_t tiles = (len + kTileBytes - 1) / kTileBytes;
    if (tiles > (uint64_t{1} << 20))
        return set_error(SBF_ERR_INVALID_ARGUMENT, "FASTX block too large for the device parser");
    // Every buffer is sized from `len` before capture (nothing allocates
    // inside the graph): newlines up to line_cap, records up to line_cap,
    // windows up to len.
    line_cap = std::max<uint64_t>(line_cap, len / 32 + 1024);
    const uint64_t max_kmers = f->kmers_of(len);
    const uint64_t max_tiles = (max_kmers + 16 + kTileKmers - 1) / kTileKmers + 1;
    int s;
    if ((s = text.ensure(len + 64)) != SBF_OK || (s = grow<uint64_t>(tile_off, tiles + 2)) != SBF_OK ||
        (s = ctl.ensure(128)) != SBF_OK || (s = grow<uint64_t>(line_end, line_cap + 1)) != SBF_OK ||
        (s = grow<DevRange>(seq, line_cap)) != SBF_OK || (s = grow<DevRange>(hdr, line_cap)) != SBF_OK ||
        (s = counts.ensure(64)) != SBF_OK || (s = g_sizes.ensure(sizeof(DevSizes))) != SBF_OK ||
        (s = g_summary.ensure(sizeof(BlockSummary))) != SBF_OK || (s = g_queue.ensure(64)) != SBF_OK ||
        (s = g_tile_rec.ensure(max_tiles * 4 + 64)) != SBF_OK ||
        (s = h_summary.ensure(sizeof(BlockSummary))) != SBF_OK)
        return s;
    if (fasta && ((s = grow<uint64_t>(line_len, line_cap + 1)) != SBF_OK ||
                  (s = grow<uint64_t>(line_hdr, line_cap + 1)) != SBF_OK ||
                  (s = comp.ensure(len + 64)) != SBF_OK))
        return s;
    if (query && (s = this->out.ensure(max_kmers + 64)) != SBF_OK) return s;
    auto* d_text = static_cast<uint8_t*>(text.ptr);
    auto* d_tiles = static_cast<uint64_t*>(tile_off.ptr);
    auto* d_ctl = static_cast<unsigned long long*>(ctl.ptr);
    auto* d_le = static_cast<uint64_t*>(line_end.ptr);
    auto* d_sizes = static_cast<DevSizes*>(g_sizes.ptr);
    auto* d_sum = static_cast<BlockSummary*>(g_summary.ptr);
    auto* d_counts = static_cast<unsigned long long*>(counts.ptr);
    uint8_t* d_hits = query ? static_cast<uint8_t*>(this->out.ptr) : nullptr;
    const uint8_t* d_base = fasta ? static_cast<const uint8_t*>(comp.ptr) : d_text;
    const uint64_t cap = line_cap;
    const unsigned fixed_grid = static_cast<unsigned>(f->sms) * 8;
    // Ragged-pass parameters: the grid phase is host-known (pointer
    // alignment), the sizes are the device's.
    const int64_t phase = query ? static_cast<int64_t>(reinterpret_cast<uintptr_t>(d_hits) & 15u)
                                : static_cast<int64_t>(reinterpret_cast<uintptr_t>(d_base) & 15u);
    TileParams p{};
    p.input = d_base;
    p.input_bytes = len;
    p.n_kmers = max_kmers;
    p.sym_base = -phase;
    p.words = f->d_words;
    p.shard_mask = static_cast<uint32_t>(f->num_shards - 1);
    p.out = d_hits;
    p.n_tiles = max_tiles;
    p.err = f->d_err;
    p.ranges = static_cast<const DevRange*>(seq.ptr);
    p.n_ranges = cap;
    p.tile_rec = static_cast<const uint32_t*>(g_tile_rec.ptr);
    p.queue = static_cast<unsigned int*>(g_queue.ptr);
    p.counts = d_counts;
    p.gen = f->gen;
    p.sizes = d_sizes;
    const int occ = f->occupancy[query ? 5 : 4];
    const unsigned tile_grid = static_cast<unsigned>(std::max<uint64_t>(
        std::min<uint64_t>(max_tiles, static_cast<uint64_t>(f->sms) * std::max(occ, 1)), 1));
    const void* tile_fn = query ? f->ks->query_ragged : f->ks->insert_ragged;

    cudaError_t e;
    if (!capture_stream &&
        (e = cudaStreamCreateWithFlags(&capture_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return cuda_fail(e, "cudaStreamCreateWithFlags");
    const cudaStream_t launch_stream = st;
    st = capture_stream;  // every call below is recorded into the graph
    if ((e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(e, "cudaStreamBeginCapture");
    }
    auto body = [&]() -> cudaError_t {
        cudaError_t r;
        if ((r = cudaMemcpyAsync(d_text, h_text, len, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (r = cudaMemsetAsync(d_ctl, 0, 128, st)) != cudaSuccess ||
            (r = cudaMemsetAsync(d_counts, 0, 16, st)) != cudaSuccess)
            return r;
        tile_newlines_kernel<<<static_cast<unsigned>(tiles), kScanThreads, 0, st>>>(d_text, len, d_tiles);
        scan_counts_kernel<<<1, 1024, 0, st>>>(d_tiles, tiles, reinterpret_cast<uint64_t*>(d_ctl));
        newline_positions_kernel<<<static_cast<unsigned>(tiles), kScanThreads, 0, st>>>(
            d_text, len, d_tiles, d_le, cap, reinterpret_cast<unsigned int*>(d_ctl + 1));
        if (!fasta) {
            fastq_records_kernel<<<fixed_grid, 256, 0, st>>>(
                d_text, d_le, 0, static_cast<DevRange*>(seq.ptr), static_cast<DevRange*>(hdr.ptr),
                reinterpret_cast<unsigned int*>(d_ctl + 1), d_ctl + 2, d_ctl, cap);
            fastq_sizes_kernel<<<1, 1, 0, st>>>(d_le, d_ctl, cap, phase, f->k, d_sizes, d_sum);
        } else {
            auto* d_len = static_cast<uint64_t*>(line_len.ptr);
            auto* d_hdrf = static_cast<uint64_t*>(line_hdr.ptr);
            fasta_lines_kernel<<<fixed_grid, 256, 0, st>>>(d_text, d_le, 0, d_len, d_hdrf, d_ctl, cap);
            scan_counts_kernel<<<1, 1024, 0, st>>>(d_len, 0, reinterpret_cast<uint64_t*>(d_ctl + 3),
                                                   d_ctl, cap);
            scan_counts_kernel<<<1, 1024, 0, st>>>(d_hdrf, 0, reinterpret_cast<uint64_t*>(d_ctl + 4),
                                                   d_ctl, cap);
            fasta_compact_kernel<<<fixed_grid, 256, 0, st>>>(d_text, d_le, 0, d_len,
                                                             static_cast<uint8_t*>(comp.ptr), d_ctl, cap);
            fasta_records_kernel<<<fixed_grid, 256, 0, st>>>(
                d_text, d_le, 0, d_len, d_hdrf, 0, static_cast<DevRange*>(seq.ptr),
                static_cast<DevRange*>(hdr.ptr), d_ctl + 5, d_ctl, cap, d_ctl + 4);
            fasta_lengths_kernel<<<fixed_grid, 256, 0, st>>>(static_cast<DevRange*>(seq.ptr), 0, 0,
                                                             d_ctl + 4, d_ctl + 3);
            fasta_sizes_kernel<<<1, 1, 0, st>>>(d_ctl, cap, len, eof ? 1 : 0, phase, f->k, d_sizes,
                                                d_sum);
        }
        if ((r = launch_tile_records_sized(p.ranges, d_sizes, p.sym_base, max_tiles,
                                           const_cast<uint32_t*>(p.tile_rec), st)) != cudaSuccess ||
            (r = cudaMemsetAsync(p.queue, 0, sizeof(unsigned int), st)) != cudaSuccess)
            return r;
        TileParams copy = p;
        void* args[] = {&copy};
        if ((r = cudaLaunchKernel(tile_fn, dim3(tile_grid), dim3(kThreads), args, f->ks->smem(query),
                                  st)) != cudaSuccess)
            return r;
        if ((r = cudaMemcpyAsync(reinterpret_cast<uint8_t*>(h_summary.p) + offsetof(BlockSummary, valid),
                                 d_counts, 16, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return r;
        return cudaMemcpyAsync(h_summary.p, d_sum, offsetof(BlockSummary, valid),
                               cudaMemcpyDeviceToHost, st);
    };
    const cudaError_t body_err = body();
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(st, &graph);
    st = launch_stream;
    if (body_err != cudaSuccess || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return cuda_fail(body_err != cudaSuccess ? body_err : e, "capturing the FASTX block graph");
    }
    // Same topology block after block: update the executable in place.
    cudaGraphExec_t& exec = graph_exec[(fasta ? 2 : 0) + (query ? 1 : 0)];
    if (exec) {
        cudaGraphExecUpdateResultInfo info{};
        if (cudaGraphExecUpdate(exec, graph, &info) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphExecDestroy(exec);
            exec = nullptr;
        }
    }
    if (!exec && (e = cudaGraphInstantiate(&exec, graph, 0)) != cudaSuccess) {
        cudaGraphDestroy(graph);
        exec = nullptr;
        return cuda_fail(e, "cudaGraphInstantiate");
    }
    cudaGraphDestroy(graph);
    if ((e = cudaGraphLaunch(exec, st)) != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
    f->launches += 2;
    return SBF_OK;
}

int PinnedBuf::ensure(size_t bytes) {
    if (bytes <= cap) return SBF_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    const size_t want = std::max<size_t>(bytes, 4096);
    if (cudaMallocHost(&p, want) != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        return set_error(SBF_ERR_RESOURCE, "cannot allocate %zu bytes of pinned memory", want);
    }
    cap = want;
    return SBF_OK;
}

void PinnedBuf::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
}

void fastq_device_release(sbf_filter* f) {
    f->fastq_block.release();
    f->fastq_ahead.release();
    if (!f->fastq) return;
    f->fastq->release();
    delete f->fastq;
    f->fastq = nullptr;
}

void FastqDevice::release() {
    for (cudaGraphExec_t& g : graph_exec) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    if (capture_stream) cudaStreamDestroy(capture_stream);
    capture_stream = nullptr;
    line_cap = 0;
    g_sizes.release();
    g_summary.release();
    g_queue.release();
    g_tile_rec.release();
    h_summary.release();
    line_len.release();
    line_hdr.release();
    comp.release();
    h_comp.release();
    text.release();
    tile_off.release();
    line_end.release();
    seq.release();
    hdr.release();
    ctl.release();
    counts.release();
    out.release();
    rec_counts.release();
    h_hits.release();
}

}  // namespace sbf
