// sbf_fastq_gpu.h -- FASTQ and FASTA blocks parsed on the GPU (sbf_fastq_gpu.cu), used
// by the FASTX entry points (sbf_fastx.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "sbf_host.h"
#include "sbf_internal.h"

namespace sbf {

// One parsed block of FASTQ text: `records` complete four-line records in
// bytes [0, consumed); `regular` is false when any record breaks the strict
// four-line layout (the caller then parses the input on the host).
// FASTA blocks are parsed the same way, except that the sequence lines are
// compacted into one buffer (d_base != d_text) and records end before the
// next '>' header.
struct FastqBlock {
    uint64_t lines = 0;
    uint64_t records = 0;     // records to process in this block
    uint64_t consumed = 0;    // text bytes of those records
    uint64_t bases = 0;       // sequence bytes of those records
    bool regular = true;
    bool compacted = false;   // FASTA: sequences live in a compacted buffer
    const uint8_t* d_text = nullptr;
    const uint8_t* d_base = nullptr;  // bytes the sequence ranges index
    uint64_t base_len = 0;            // bytes of d_base covered by the records
    const DevRange* d_seq = nullptr;  // sequence of each record (offsets into d_base)
    const DevRange* d_hdr = nullptr;  // header without '@' / '>' (offsets into the text)
};

// BlockSummary::flags bits.
enum : uint64_t { kBlockIrregular = 1u, kBlockLineOverflow = 2u };

// What one block replayed as a CUDA graph reports back (one download).
struct BlockSummary {
    uint64_t lines;       // newlines in the block
    uint64_t flags;       // kIrregular / kLineOverflow bits
    uint64_t bases;       // sequence bytes of the records processed
    uint64_t consumed;    // text bytes of the records processed
    uint64_t records;     // records processed
    uint64_t lines_used;  // lines of the records processed
    uint64_t valid, positive;
};

struct FastqDevice {
    DevBuf text, tile_off, line_end, seq, hdr, ctl, counts, out, rec_counts;
    DevBuf line_len, line_hdr, comp;  // FASTA line tables and compacted sequence
    DevBuf g_sizes, g_summary, g_queue, g_tile_rec;  // graph replay
    PinnedBuf h_hits, h_comp, h_summary;
    // One executable per (FASTA?, query?): blocks of one kind update theirs in
    // place; a different kind never forces a re-instantiation.
    cudaGraphExec_t graph_exec[4] = {nullptr, nullptr, nullptr, nullptr};
    // Blocks are captured on this stream (the caller's may be the legacy
    // default stream, which cannot be captured) and launched on the caller's.
    cudaStream_t capture_stream = nullptr;
    uint64_t line_cap = 0;  // line_end entries the graph path may write
    // Filled by run() when record views are wanted.
    std::vector<DevRange> h_seq, h_hdr;
    std::vector<unsigned long long> h_valid, h_pos;

    // Uploads and parses h_text[0, len) (which starts at a record start).
    int parse(sbf_filter* f, const uint8_t* h_text, uint64_t len, cudaStream_t st, FastqBlock* out);
    // FASTA: h_text starts at a '>' header; with `eof` the last record is
    // complete, otherwise it is left for the next block (records = 0 when the
    // block holds no complete record).
    int parse_fasta(sbf_filter* f, const uint8_t* h_text, uint64_t len, bool eof, cudaStream_t st,
                    FastqBlock* out);
    // Uploads h_text and locates its newlines (line_end[0, *n_lines)).
    int scan_lines(sbf_filter* f, const uint8_t* h_text, uint64_t len, cudaStream_t st,
                   uint64_t* n_lines);
    // Inserts or queries the block's records (one ragged pass); valid and
    // positive windows are returned, and with want_views the per-record
    // table, counts and hits are copied to the host (h_* members).
    int run(sbf_filter* f, bool query, const FastqBlock& b, cudaStream_t st, bool want_views,
            uint64_t* valid, uint64_t* positive);
    // Upload, parse and insert / query one FASTQ (fasta = false) or FASTA
    // block as one CUDA graph with a single synchronisation: the record count,
    // sequence length and regularity are found and used on the device, and
    // an irregular block or one whose newlines overflow line_end runs no
    // insert or query (the caller retries or parses on the host).  Without
    // per-record views only; needs kernels compiled into the library.
    int run_block_graph(sbf_filter* f, bool query, bool fasta, const uint8_t* h_text,
                        uint64_t len, bool eof, cudaStream_t st, BlockSummary* out);
    // The same in two halves: launch returns once the graph is queued (the
    // host text must stay untouched until finish), finish waits for it and
    // fills the summary.
    int launch_block_graph(sbf_filter* f, bool query, bool fasta, const uint8_t* h_text,
                           uint64_t len, bool eof, cudaStream_t st);
    int finish_block_graph(sbf_filter* f, cudaStream_t st, BlockSummary* out);
    static bool graph_usable(const sbf_filter* f);
    const uint8_t* hits_host() const { return static_cast<const uint8_t*>(h_hits.p); }
    // FASTA sequences for record views (filled by run() with want_views).
    const uint8_t* comp_host() const { return static_cast<const uint8_t*>(h_comp.p); }
    void release();
};

void fastq_device_release(sbf_filter* f);

}  // namespace sbf
