// sbf_fastq_gpu.h -- FASTQ blocks parsed on the GPU (sbf_fastq_gpu.cu), used
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
struct FastqBlock {
    uint64_t lines = 0;
    uint64_t records = 0;
    uint64_t consumed = 0;
    uint64_t bases = 0;
    bool regular = true;
    const uint8_t* d_text = nullptr;
    const DevRange* d_seq = nullptr;  // sequence line of each record (block offsets)
    const DevRange* d_hdr = nullptr;  // header without '@'
};

struct FastqDevice {
    DevBuf text, tile_off, line_end, seq, hdr, ctl, counts, out, rec_counts;
    PinnedBuf h_hits;
    // Filled by run() when record views are wanted.
    std::vector<DevRange> h_seq, h_hdr;
    std::vector<unsigned long long> h_valid, h_pos;

    // Uploads and parses h_text[0, len) (which starts at a record start).
    int parse(sbf_filter* f, const uint8_t* h_text, uint64_t len, cudaStream_t st, FastqBlock* out);
    // Inserts or queries the block's records (one ragged pass); valid and
    // positive windows are returned, and with want_views the per-record
    // table, counts and hits are copied to the host (h_* members).
    int run(sbf_filter* f, bool query, const FastqBlock& b, cudaStream_t st, bool want_views,
            uint64_t* valid, uint64_t* positive);
    const uint8_t* hits_host() const { return static_cast<const uint8_t*>(h_hits.p); }
    void release();
};

void fastq_device_release(sbf_filter* f);

}  // namespace sbf
