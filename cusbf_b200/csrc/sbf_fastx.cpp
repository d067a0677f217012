// sbf_fastx.cpp -- streaming FASTA/FASTQ parsing and the FASTX entry points.
//
// Parsing rules follow the reference reader (include/cusbf/Fastx.hpp:297-462
// of tdortman/cuSBF):
//   * blank lines before a header are skipped; a trailing '\r' is trimmed;
//   * the first header fixes the format ('>' FASTA, '@' FASTQ); a header of
//     the other kind is an error; anything else is an error;
//   * FASTA sequence lines run until the next line starting with '>';
//   * FASTQ sequence lines run until a line starting with '+', then quality
//     lines are read until their total length reaches the sequence length
//     (longer or shorter is an error; end of input before '+' is an error);
//   * error locations are "source:line:column" (Fastx.hpp:268-289).
// Chunking follows run_fastx_pipeline (detail/fastx_pipeline_core.cuh:33-122)
// and fastx_chunk_reached_staging_budget (detail/fastx_chunk.cuh:97-127):
// a chunk is flushed once its estimated device staging reaches
// fill_fraction * (free memory - 64 MiB), or after every record when that
// budget is 0.  Each flushed chunk is one record batch, so k-mers never span
// records.  Unlike the reference reader, lines are scanned with memchr over a
// large buffer instead of std::getline.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/sbf_b200.h"
#include "sbf_fastq_gpu.h"
#include "sbf_host.h"

namespace sbf {

namespace {

class LineReader {
   public:
    LineReader(sbf_read_fn read, void* user) : read_(read), user_(user), buf_(1 << 22) {}

    // Next line without its '\n' (and without a trailing '\r').  Returns 1
    // with a line, 0 at end of input, -1 on a read error.
    int next(std::string& line) {
        line.clear();
        for (;;) {
            if (pos_ == end_) {
                if (eof_) return line.empty() && !partial_ ? 0 : finish(line);
                const int64_t n = read_(user_, buf_.data(), buf_.size());
                if (n < 0) return -1;
                if (n == 0) {
                    eof_ = true;
                    continue;
                }
                pos_ = 0;
                end_ = static_cast<size_t>(n);
            }
            const char* p = buf_.data() + pos_;
            const void* nl = std::memchr(p, '\n', end_ - pos_);
            if (nl) {
                const size_t len = static_cast<const char*>(nl) - p;
                line.append(p, len);
                pos_ += len + 1;
                partial_ = false;
                trim(line);
                return 1;
            }
            line.append(p, end_ - pos_);
            partial_ = true;
            pos_ = end_;
        }
    }

   private:
    int finish(std::string& line) {
        partial_ = false;
        trim(line);
        return 1;
    }
    static void trim(std::string& line) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
    }

    sbf_read_fn read_;
    void* user_;
    std::vector<char> buf_;
    size_t pos_ = 0, end_ = 0;
    bool eof_ = false;
    bool partial_ = false;
};

enum class Format { unknown, fasta, fastq };

class FastxParser {
   public:
    // line_base: lines of the input already consumed before `read`'s first
    // byte (error locations count from the start of the whole input).
    FastxParser(sbf_read_fn read, void* user, std::string source, uint64_t line_base = 0)
        : lines_(read, user), source_(std::move(source)), line_no_(line_base) {}

    // 1 = record, 0 = end of input, or an sbf_status error (negated).
    int next(std::string& header, std::string& seq) {
        header.clear();
        seq.clear();
        std::string* hdr = nullptr;
        if (!pending_.empty()) {
            header.swap(pending_);
            pending_.clear();
            hdr = &header;
        } else {
            for (;;) {
                const int r = lines_.next(line_);
                if (r < 0) return -io_error();
                if (r == 0) return 0;
                ++line_no_;
                if (!line_.empty()) break;
            }
            header.swap(line_);
            hdr = &header;
        }
        const char tag = hdr->front();
        if (format_ == Format::unknown) {
            if (tag == '>')
                format_ = Format::fasta;
            else if (tag == '@')
                format_ = Format::fastq;
            else
                return -parse_error("expected FASTA or FASTQ header", 1);
        }
        const char expect = format_ == Format::fasta ? '>' : '@';
        if (tag != expect) return -parse_error("mixed FASTA and FASTQ records are not supported", 1);
        hdr->erase(0, 1);
        return format_ == Format::fasta ? read_fasta(seq) : read_fastq(seq);
    }

   private:
    int read_fasta(std::string& seq) {
        for (;;) {
            const int r = lines_.next(line_);
            if (r < 0) return -io_error();
            if (r == 0) return 1;
            ++line_no_;
            if (!line_.empty() && line_.front() == '>') {
                pending_.swap(line_);
                return 1;
            }
            seq += line_;
        }
    }

    int read_fastq(std::string& seq) {
        for (;;) {
            const int r = lines_.next(line_);
            if (r < 0) return -io_error();
            if (r == 0) {
                const uint32_t col = line_.empty() ? 1 : static_cast<uint32_t>(line_.size());
                return -parse_error("unterminated FASTQ record: missing '+' separator", col);
            }
            ++line_no_;
            if (!line_.empty() && line_.front() == '+') break;
            seq += line_;
        }
        // Qualities until their length reaches the sequence length.
        const uint64_t expect = seq.size();
        uint64_t qual = 0;
        uint32_t short_col = 1;
        while (qual < expect) {
            const int r = lines_.next(line_);
            if (r < 0) return -io_error();
            if (r == 0) break;
            ++line_no_;
            short_col = line_.empty() ? 1 : static_cast<uint32_t>(line_.size() + 1);
            qual += line_.size();
            if (qual > expect) {
                const uint64_t before = qual - line_.size();
                const uint64_t idx = expect > before ? expect - before : line_.size();
                const uint32_t col = line_.empty()
                                         ? 1
                                         : static_cast<uint32_t>(std::min<uint64_t>(idx, line_.size() - 1) + 1);
                return -parse_error("FASTQ quality length exceeds sequence length", col);
            }
        }
        if (qual == expect) return 1;
        return -parse_error("FASTQ quality length does not match sequence length", short_col);
    }

    int parse_error(const char* what, uint32_t col) {
        set_error_location(source_.c_str(), static_cast<uint32_t>(line_no_), col);
        return set_error(SBF_ERR_FASTX_PARSE, "%s:%llu:%u: %s", source_.c_str(),
                         static_cast<unsigned long long>(line_no_), col, what);
    }
    int io_error() {
        return set_error(SBF_ERR_IO, "Failed to read FASTA/FASTQ input from %s", source_.c_str());
    }

    LineReader lines_;
    std::string source_;
    std::string line_, pending_;
    Format format_ = Format::unknown;
    uint64_t line_no_ = 0;
};

// Staging budget (detail/fastx_chunk.cuh:97-107).
size_t staging_budget(double fill_fraction) {
    if (fill_fraction <= 0.0) return 0;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    const size_t slack = size_t{64} << 20;
    const size_t avail = free_b > slack ? free_b - slack : 0;
    const double b = static_cast<double>(avail) * fill_fraction;
    return b <= 0 ? 0 : static_cast<size_t>(b);
}

size_t host_chunk_limit() {
    if (const char* v = std::getenv("SBF_FASTX_MAX_HOST_CHUNK_MB")) {
        const long long mb = std::strtoll(v, nullptr, 10);
        if (mb > 0) return static_cast<size_t>(mb) << 20;
    }
    return size_t{1} << 30;
}

// Whether the chunk's estimated staging reaches the budget
// (fastx_chunk_reached_staging_budget, detail/fastx_chunk.cuh:110-127).
bool should_flush(bool query, size_t budget, uint64_t raw, uint64_t records, uint32_t k,
                  uint32_t width) {
    if (raw == 0) return false;
    if (budget == 0) return true;
    const uint64_t norm = raw + records * 2 * width;
    uint64_t staging = norm;
    if (query) staging += norm / width < k ? 0 : norm / width - k + 1;
    return staging >= budget || raw >= host_chunk_limit();
}

struct Chunk {
    std::string seq;
    std::vector<sbf_record_range> ranges;
    std::vector<std::string> headers;
    uint64_t first_index = 0;
    void clear() {
        seq.clear();
        ranges.clear();
        headers.clear();
    }
};

struct QueryCtx {
    const Chunk* chunk;
    sbf_fastx_record_cb consume;
    void* user;
};

int chunk_record_cb(void* u, const sbf_record_view* v) {
    auto* ctx = static_cast<QueryCtx*>(u);
    const std::string& h = ctx->chunk->headers[v->record_index];
    sbf_fastx_record_view fv{ctx->chunk->first_index + v->record_index,
                             h.data(),
                             h.size(),
                             v->sequence,
                             v->sequence_bytes,
                             v->queried_bases,
                             v->queried_kmers,
                             v->positive_kmers,
                             v->hits,
                             v->n_hits};
    return ctx->consume(ctx->user, &fv);
}

// Host parsing (FastxReader semantics) of the input from `read`, whose first
// byte starts line line_base + 1 and record index_base; reports are added to
// `it` / `qt`.
int run_fastx_host(sbf_filter* f, bool query, sbf_read_fn read, void* ruser, const char* source,
                   double fill_fraction, sbf_stream_t stream, sbf_insert_report& it,
                   sbf_query_report& qt, sbf_fastx_record_cb consume, void* cuser,
                   uint64_t line_base, uint64_t index_base) {
    FastxParser parser(read, ruser, source ? source : "<stream>", line_base);
    const size_t budget = staging_budget(fill_fraction);
    Chunk chunk;
    chunk.first_index = index_base;
    uint64_t next_index = index_base;
    std::string header, seq;
    auto flush = [&]() -> int {
        if (chunk.ranges.empty()) return SBF_OK;
        if (query) {
            sbf_query_report r{};
            QueryCtx ctx{&chunk, consume, cuser};
            const int s = query_record_batch_impl(f, chunk.seq.data(), chunk.seq.size(),
                                                  chunk.ranges.data(), chunk.ranges.size(), stream,
                                                  &r, consume ? chunk_record_cb : nullptr, &ctx);
            if (s != SBF_OK) return s;
            qt.records_queried += r.records_queried;
            qt.queried_bases += r.queried_bases;
            qt.queried_kmers += r.queried_kmers;
            qt.positive_kmers += r.positive_kmers;
        } else {
            sbf_insert_report r{};
            const int s = insert_record_batch_impl(f, chunk.seq.data(), chunk.seq.size(),
                                                   chunk.ranges.data(), chunk.ranges.size(),
                                                   stream, &r);
            if (s != SBF_OK) return s;
            it.records_indexed += r.records_indexed;
            it.indexed_bases += r.indexed_bases;
            it.inserted_kmers += r.inserted_kmers;
        }
        chunk.clear();
        chunk.first_index = next_index;
        return SBF_OK;
    };
    for (;;) {
        const int r = parser.next(header, seq);
        if (r < 0) return -r;
        if (r == 0) break;
        chunk.ranges.push_back(sbf_record_range{chunk.seq.size(), seq.size()});
        chunk.seq += seq;
        if (query && consume) chunk.headers.push_back(header);
        ++next_index;
        if (should_flush(query, budget, chunk.seq.size(), chunk.ranges.size(), f->k, f->width)) {
            const int s = flush();
            if (s != SBF_OK) return s;
        }
    }
    return flush();
}

// Serves `data` first, then the rest of the input from `inner`.
struct PrefixReader {
    const char* data;
    size_t len, pos;
    sbf_read_fn inner;
    void* inner_user;
    static int64_t read(void* u, char* buf, uint64_t cap) {
        auto* r = static_cast<PrefixReader*>(u);
        if (r->pos < r->len) {
            const size_t n = std::min<size_t>(cap, r->len - r->pos);
            std::memcpy(buf, r->data + r->pos, n);
            r->pos += n;
            return static_cast<int64_t>(n);
        }
        return r->inner(r->inner_user, buf, cap);
    }
};

bool device_fastq_enabled() {
    const char* v = std::getenv("SBF_FASTX_PARSER");
    return !(v && std::strcmp(v, "host") == 0);
}

// Blocks without per-record views run as one CUDA graph each
// (SBF_FASTX_GRAPH=0 runs them as stream launches).
bool fastx_graph_enabled() {
    const char* v = std::getenv("SBF_FASTX_GRAPH");
    return !(v && std::strcmp(v, "0") == 0);
}

// FASTQ blocks on the graph path read the next block while the device
// works on the current one (SBF_FASTQ_READ_AHEAD=0 reads them in turn).
bool fastq_read_ahead_enabled() {
    const char* v = std::getenv("SBF_FASTQ_READ_AHEAD");
    return !(v && std::strcmp(v, "0") == 0);
}

// Room in front of each FASTQ block buffer for the previous block's
// unconsumed tail (less than one record); a longer tail hands the rest of
// the input to the host parser.
constexpr uint64_t kTailRoom = uint64_t{32} << 20;

uint64_t fastq_block_bytes() {
    if (const char* v = std::getenv("SBF_FASTQ_BLOCK_BYTES")) {
        const long long b = std::strtoll(v, nullptr, 10);
        if (b >= 4096) return static_cast<uint64_t>(b);
    }
    return uint64_t{256} << 20;
}

// FASTQ and FASTA input through the GPU parsers in blocks of complete
// records (FASTQ: strictly four-line records; FASTA: records end before the
// next '>' header, and a record longer than the block grows it); falls back
// to run_fastx_host for the rest of the input at the first block that is
// anything else, so results and errors are always the host parser's.
int run_fastx(sbf_filter* f, bool query, sbf_read_fn read, void* ruser, const char* source,
              double fill_fraction, sbf_stream_t stream, sbf_insert_report* irep,
              sbf_query_report* qrep, sbf_fastx_record_cb consume, void* cuser) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    if (!read) return set_error(SBF_ERR_INVALID_ARGUMENT, "read callback is null");
    sbf_insert_report it{0, 0, 0};
    sbf_query_report qt{0, 0, 0, 0};
    auto finish = [&](int s) -> int {
        if (s != SBF_OK) return s;
        if (irep) *irep = it;
        if (qrep) *qrep = qt;
        return SBF_OK;
    };
    // The GPU parsers feed a ragged pass over the raw text, whose symbol grid
    // is the buffer's: multi-byte symbols (DNA triplets) need each record
    // padded to a symbol boundary, which the host path's normalisation does.
    if (!device_fastq_enabled() || f->width != 1)
        return finish(run_fastx_host(f, query, read, ruser, source, fill_fraction, stream, it, qt,
                                     consume, cuser, 0, 0));
    if (!f->fastq) f->fastq = new FastqDevice();
    FastqDevice& dev = *f->fastq;
    uint64_t cap = fastq_block_bytes();
    const uint64_t kMaxBlockBytes = uint64_t{8} << 30;  // FASTA records up to this size
    PinnedBuf& buf = f->fastq_block;
    int s = buf.ensure(kTailRoom + cap + 1);
    if (s != SBF_OK) return s;
    auto* text = static_cast<char*>(buf.p);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    uint64_t len = 0, line_base = 0, index_base = 0;
    bool eof = false;
    auto fallback = [&](uint64_t valid_len) -> int {
        PrefixReader pr{text, valid_len, 0, read, ruser};
        return finish(run_fastx_host(f, query, &PrefixReader::read, &pr, source, fill_fraction,
                                     stream, it, qt, consume, cuser, line_base, index_base));
    };
    for (;;) {
        while (!eof && len < cap) {
            const int64_t n = read(ruser, text + len, cap - len);
            if (n < 0)
                return set_error(SBF_ERR_IO, "Failed to read FASTA/FASTQ input from %s",
                                 source ? source : "<stream>");
            if (n == 0)
                eof = true;
            else
                len += static_cast<uint64_t>(n);
        }
        if (len == 0) break;
        const bool fastq = text[0] == '@';
        if (!fastq && text[0] != '>') return fallback(len);  // blank lines, or not FASTX
        uint64_t parse_len = len;
        if (eof && text[len - 1] != '\n') {
            text[len] = '\n';  // the last line ends at end of input
            parse_len = len + 1;
        }
        const bool views = query && consume;
        if (fastq && !views && fastx_graph_enabled() && fastq_read_ahead_enabled() &&
            FastqDevice::graph_usable(f)) {
            // The block runs as one graph while the next block is read into
            // the other pinned buffer, behind kTailRoom bytes that then take
            // this block's unconsumed tail, so the next block is contiguous.
            BlockSummary g;
            s = dev.launch_block_graph(f, query, false, reinterpret_cast<const uint8_t*>(text),
                                       parse_len, eof, st);
            if (s != SBF_OK) return s;
            char* ahead = nullptr;
            uint64_t nb = 0;
            bool eof2 = eof;
            int rs = SBF_OK;
            if (!eof) {
                const char* a0 = static_cast<const char*>(f->fastq_block.p);
                const bool in_block = text >= a0 && text < a0 + f->fastq_block.cap;
                PinnedBuf& other = in_block ? f->fastq_ahead : f->fastq_block;
                rs = other.ensure(kTailRoom + cap + 1);
                if (rs == SBF_OK) ahead = static_cast<char*>(other.p) + kTailRoom;
                while (rs == SBF_OK && !eof2 && nb < cap) {
                    const int64_t n = read(ruser, ahead + nb, cap - nb);
                    if (n < 0)
                        rs = set_error(SBF_ERR_IO, "Failed to read FASTA/FASTQ input from %s",
                                       source ? source : "<stream>");
                    else if (n == 0)
                        eof2 = true;
                    else
                        nb += static_cast<uint64_t>(n);
                }
            }
            if ((s = dev.finish_block_graph(f, st, &g)) != SBF_OK) return s;
            if (rs != SBF_OK) return rs;
            while (g.flags & kBlockLineOverflow) {  // line table grown: run the block again
                s = dev.run_block_graph(f, query, false, reinterpret_cast<const uint8_t*>(text),
                                        parse_len, eof, st, &g);
                if (s != SBF_OK) return s;
            }
            // The host parser takes over from `from` with the read-ahead bytes
            // in front of the rest of the input.
            auto fallback_from = [&](uint64_t from) -> int {
                std::string pre(text + from, len - from);
                if (nb) pre.append(ahead, nb);
                PrefixReader pr{pre.data(), pre.size(), 0, read, ruser};
                return finish(run_fastx_host(f, query, &PrefixReader::read, &pr, source,
                                             fill_fraction, stream, it, qt, consume, cuser,
                                             line_base, index_base));
            };
            // An insert of the records before a fallback is repeated by the
            // host path, which ORs the same bits again.
            if ((g.flags & kBlockIrregular) || g.records == 0 || (eof && g.consumed < parse_len))
                return fallback_from(0);
            if (query) {
                qt.records_queried += g.records;
                qt.queried_bases += g.bases;
                qt.queried_kmers += g.valid;
                qt.positive_kmers += g.positive;
            } else {
                it.records_indexed += g.records;
                it.indexed_bases += g.bases;
                it.inserted_kmers += g.valid;
            }
            index_base += g.records;
            line_base += g.lines_used;
            const uint64_t consumed = std::min<uint64_t>(g.consumed, len);
            const uint64_t tail = len - consumed;
            if (eof) {
                std::memmove(text, text + consumed, tail);
                len = tail;
                if (len == 0) break;
                continue;
            }
            if (tail > kTailRoom) return fallback_from(consumed);
            std::memcpy(ahead - tail, text + consumed, tail);
            text = ahead - tail;
            len = tail + nb;
            eof = eof2;
            if (eof && len == 0) break;
            continue;
        }
        if (!views && fastx_graph_enabled() && FastqDevice::graph_usable(f)) {
            BlockSummary g;
            s = dev.run_block_graph(f, query, !fastq, reinterpret_cast<const uint8_t*>(text),
                                    parse_len, eof, st, &g);
            if (s != SBF_OK) return s;
            if (g.flags & kBlockLineOverflow) continue;  // line table grown: run the block again
            if (fastq) {
                // An insert of the records before a fallback is repeated by
                // the host path, which ORs the same bits again.
                if ((g.flags & kBlockIrregular) || g.records == 0 || (eof && g.consumed < parse_len))
                    return fallback(len);
            } else {
                if (g.flags & kBlockIrregular) return fallback(len);
                if (g.records == 0) {
                    if (eof || cap >= kMaxBlockBytes) return fallback(len);
                    PinnedBuf bigger;
                    if ((s = bigger.ensure(2 * cap + 1)) != SBF_OK) return fallback(len);
                    std::memcpy(bigger.p, text, len);
                    buf.release();
                    buf = bigger;
                    bigger.p = nullptr;
                    text = static_cast<char*>(buf.p);
                    cap *= 2;
                    continue;
                }
            }
            if (query) {
                qt.records_queried += g.records;
                qt.queried_bases += g.bases;
                qt.queried_kmers += g.valid;
                qt.positive_kmers += g.positive;
            } else {
                it.records_indexed += g.records;
                it.indexed_bases += g.bases;
                it.inserted_kmers += g.valid;
            }
            index_base += g.records;
            line_base += g.lines_used;
            const uint64_t consumed = std::min<uint64_t>(g.consumed, len);
            std::memmove(text, text + consumed, len - consumed);
            len -= consumed;
            if (eof && len == 0) break;
            continue;
        }
        FastqBlock b;
        if (fastq) {
            s = dev.parse(f, reinterpret_cast<const uint8_t*>(text), parse_len, st, &b);
            if (s != SBF_OK) return s;
            if (!b.regular || b.records == 0 || (eof && b.consumed < parse_len)) return fallback(len);
        } else {
            s = dev.parse_fasta(f, reinterpret_cast<const uint8_t*>(text), parse_len, eof, st, &b);
            if (s != SBF_OK) return s;
            if (!b.regular) return fallback(len);
            if (b.records == 0) {
                // One record longer than the block: grow the block and read on.
                if (eof || cap >= kMaxBlockBytes) return fallback(len);
                PinnedBuf bigger;
                if ((s = bigger.ensure(2 * cap + 1)) != SBF_OK) return fallback(len);
                std::memcpy(bigger.p, text, len);
                buf.release();
                buf = bigger;
                bigger.p = nullptr;
                text = static_cast<char*>(buf.p);
                cap *= 2;
                continue;
            }
        }
        uint64_t valid = 0, positive = 0;
        if ((s = dev.run(f, query, b, st, views, &valid, &positive)) != SBF_OK) return s;
        if (query) {
            qt.records_queried += b.records;
            qt.queried_bases += b.bases;
            qt.queried_kmers += valid;
            qt.positive_kmers += positive;
        } else {
            it.records_indexed += b.records;
            it.indexed_bases += b.bases;
            it.inserted_kmers += valid;
        }
        if (views) {
            const char* seq_base =
                b.compacted ? reinterpret_cast<const char*>(dev.comp_host()) : text;
            for (uint64_t r = 0; r < b.records; ++r) {
                const DevRange sq = dev.h_seq[r], hd = dev.h_hdr[r];
                sbf_fastx_record_view v{index_base + r,
                                        text + hd.offset,
                                        hd.bytes,
                                        seq_base + sq.offset,
                                        sq.bytes,
                                        sq.bytes,
                                        dev.h_valid[r],
                                        dev.h_pos[r],
                                        dev.hits_host() + sq.offset,
                                        sq.bytes >= f->k ? sq.bytes - f->k + 1 : 0};
                if (consume(cuser, &v) != 0)
                    return set_error(SBF_ERR_ABORTED, "record consumer aborted the query");
            }
        }
        index_base += b.records;
        line_base += fastq ? 4 * b.records : b.lines;
        const uint64_t consumed = std::min<uint64_t>(b.consumed, len);
        std::memmove(text, text + consumed, len - consumed);
        len -= consumed;
        if (eof && len == 0) break;
    }
    return finish(SBF_OK);
}

// An open FASTA/FASTQ file.  gzip input (and anything that is not a regular
// file) goes through zlib; an uncompressed regular file is read with pread()
// straight into the caller's buffer, on several threads for large reads, so a
// 256 MiB block costs one page-cache copy instead of zlib's buffered two.
struct FastxFile {
    gzFile gz = nullptr;
    int fd = -1;
    uint64_t pos = 0;
    uint64_t size = 0;
};

constexpr uint64_t kParallelReadBytes = uint64_t{8} << 20;  // below this, one pread
constexpr unsigned kReadThreads = 8;

// Reads buf[0, n) from offset `at`; false on an I/O error or early end.
bool pread_all(int fd, char* buf, uint64_t n, uint64_t at) {
    while (n) {
        const ssize_t r = ::pread(fd, buf, std::min<uint64_t>(n, uint64_t{1} << 30),
                                  static_cast<off_t>(at));
        if (r <= 0) return false;
        buf += r;
        at += static_cast<uint64_t>(r);
        n -= static_cast<uint64_t>(r);
    }
    return true;
}

int64_t file_read(void* user, char* buf, uint64_t cap) {
    auto* f = static_cast<FastxFile*>(user);
    if (f->gz) {
        const unsigned chunk = static_cast<unsigned>(std::min<uint64_t>(cap, 1u << 30));
        const int n = gzread(f->gz, buf, chunk);
        return n < 0 ? -1 : n;
    }
    const uint64_t n = f->pos < f->size ? std::min<uint64_t>(cap, f->size - f->pos) : 0;
    if (n == 0) return 0;
    bool ok = true;
    if (n < kParallelReadBytes) {
        ok = pread_all(f->fd, buf, n, f->pos);
    } else {
        const uint64_t per = (n + kReadThreads - 1) / kReadThreads;
        std::vector<std::thread> pool;
        std::vector<char> good(kReadThreads, 1);
        try {
            for (unsigned t = 0; t < kReadThreads; ++t) {
                const uint64_t a = t * per, b = std::min<uint64_t>(n, a + per);
                if (a >= b) break;
                pool.emplace_back([&, t, a, b] { good[t] = pread_all(f->fd, buf + a, b - a, f->pos + a); });
            }
        } catch (...) {
            for (auto& th : pool) th.join();
            return pread_all(f->fd, buf, n, f->pos) ? (f->pos += n, static_cast<int64_t>(n)) : -1;
        }
        for (auto& th : pool) th.join();
        for (char g : good) ok = ok && g;
    }
    if (!ok) return -1;
    f->pos += n;
    return static_cast<int64_t>(n);
}

// Opens a plain or gzip file.
int open_fastx(const char* path, FastxFile* out) {
    if (!path) return set_error(SBF_ERR_INVALID_ARGUMENT, "path is null");
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0) return set_error(SBF_ERR_IO, "Failed to open FASTA/FASTQ file: %s", path);
    struct stat st {};
    unsigned char magic[2] = {0, 0};
    const bool regular = ::fstat(fd, &st) == 0 && S_ISREG(st.st_mode);
    const bool gzip = regular && st.st_size >= 2 && ::pread(fd, magic, 2, 0) == 2 &&
                      magic[0] == 0x1f && magic[1] == 0x8b;
    if (regular && !gzip) {
        out->fd = fd;
        out->size = static_cast<uint64_t>(st.st_size);
        return SBF_OK;
    }
    ::close(fd);
    gzFile g = gzopen(path, "rb");
    if (!g) return set_error(SBF_ERR_IO, "Failed to open FASTA/FASTQ file: %s", path);
    gzbuffer(g, 1 << 20);
    out->gz = g;
    return SBF_OK;
}

void close_fastx(FastxFile& f) {
    if (f.gz) gzclose(f.gz);
    if (f.fd >= 0) ::close(f.fd);
    f = FastxFile{};
}

}  // namespace

}  // namespace sbf

using namespace sbf;

extern "C" int sbf_fastx_scan(sbf_read_fn read, void* ruser, const char* source_name,
                              sbf_fastx_scan_cb consume, void* user, uint64_t* records_out) {
    if (!read || !consume) return set_error(SBF_ERR_INVALID_ARGUMENT, "null callback");
    FastxParser parser(read, ruser, source_name ? source_name : "<stream>");
    std::string header, seq;
    uint64_t n = 0;
    for (;;) {
        const int r = parser.next(header, seq);
        if (r < 0) return -r;
        if (r == 0) break;
        if (consume(user, n, header.data(), header.size(), seq.data(), seq.size()) != 0)
            return set_error(SBF_ERR_ABORTED, "record consumer aborted the scan");
        ++n;
    }
    if (records_out) *records_out = n;
    return SBF_OK;
}

extern "C" int sbf_fastx_scan_file(const char* path, sbf_fastx_scan_cb consume, void* user,
                                   uint64_t* records_out) {
    FastxFile g;
    const int o = open_fastx(path, &g);
    if (o != SBF_OK) return o;
    const int s = sbf_fastx_scan(file_read, &g, path, consume, user, records_out);
    close_fastx(g);
    return s;
}

extern "C" int sbf_insert_fastx(sbf_filter_t* f, sbf_read_fn read, void* ruser,
                                const char* source_name, double fill_fraction,
                                sbf_stream_t stream, sbf_insert_report* report) {
    return run_fastx(f, false, read, ruser, source_name, fill_fraction, stream, report, nullptr,
                     nullptr, nullptr);
}

extern "C" int sbf_insert_fastx_file(sbf_filter_t* f, const char* path, double fill_fraction,
                                     sbf_stream_t stream, sbf_insert_report* report) {
    FastxFile g;
    const int o = open_fastx(path, &g);
    if (o != SBF_OK) return o;
    const int s = run_fastx(f, false, file_read, &g, path, fill_fraction, stream, report, nullptr,
                            nullptr, nullptr);
    close_fastx(g);
    return s;
}

extern "C" int sbf_query_fastx(const sbf_filter_t* f, sbf_read_fn read, void* ruser,
                               const char* source_name, double fill_fraction, sbf_stream_t stream,
                               sbf_query_report* report, sbf_fastx_record_cb consume,
                               void* user) {
    return run_fastx(const_cast<sbf_filter*>(f), true, read, ruser, source_name, fill_fraction,
                     stream, nullptr, report, consume, user);
}

extern "C" int sbf_query_fastx_file(const sbf_filter_t* f, const char* path, double fill_fraction,
                                    sbf_stream_t stream, sbf_query_report* report,
                                    sbf_fastx_record_cb consume, void* user) {
    FastxFile g;
    const int o = open_fastx(path, &g);
    if (o != SBF_OK) return o;
    const int s = run_fastx(const_cast<sbf_filter*>(f), true, file_read, &g, path, fill_fraction,
                            stream, nullptr, report, consume, user);
    close_fastx(g);
    return s;
}
