// sbf_internal.h -- types shared by the kernels and the C-ABI layer.
#pragma once

#ifndef __CUDACC_RTC__
#include <cuda_runtime.h>

#include <cstdint>
#endif

namespace sbf {

// Launch geometry of the tile kernels.
constexpr int kThreads = 256;                          // threads per CTA
constexpr int kStrip = 32;                             // consecutive k-mers per thread
constexpr int kTileKmers = kThreads * kStrip;          // k-mers per tile (8192)
constexpr int kStripWords = kStrip / 16 + 2;           // code words one strip reads
constexpr int kCodeWords = (kThreads - 1) * (kStrip / 16) + kStripWords;  // per tile
constexpr int kStageBytes = kCodeWords * 16 + 64;      // staged input bytes per buffer
constexpr int kSlots = 10;                             // query shard slots per thread
constexpr int kOverflow = 6;                           // deferred shard loads per thread
constexpr int kQuerySlotBytes = kSlots * kThreads * 32 + kOverflow * kThreads * 4;
constexpr int kFlushSlots = 8;                         // insert bulk-reduce staging slots
constexpr int kInsertSlotBytes = kFlushSlots * kThreads * 32;  // dynamic smem of inserts

// A record of a ragged launch: bytes [offset, offset + bytes) of the input.
// Same layout as sbf_record_range of the C ABI.
struct DevRange {
    uint64_t offset;
    uint64_t bytes;
};

// Configuration of the runtime-parameterised kernels (sbf_generic.cu), used
// for every configuration and alphabet that has no specialised kernel.
struct GenericCfg {
    uint32_t k, s, m, h;
    uint32_t bits;      // bits per packed symbol
    uint32_t width;     // input bytes per symbol
    uint32_t alphabet;  // SBF_ALPHABET_*
};

// Sizes of a ragged launch that are known only on the device: a FASTX block
// parsed on the GPU and replayed as one CUDA graph finds its record count and
// sequence length on the device, so the graph's launches read them here.
struct DevSizes {
    uint64_t input_bytes;
    uint64_t n_kmers;
    uint64_t n_tiles;   // 0 skips the pass
    uint64_t n_ranges;
};

// One launch of a tile kernel.  Grid position g of tile n is
// g = n * kTileKmers + (0 .. kTileKmers-1); it holds window (k-mer)
// i = g + sym_base, and symbol i is the first base of that window.
struct TileParams {
    const uint8_t* input;    // device bytes (ASCII) or dense words viewed as bytes
    uint64_t input_bytes;    // readable bytes at `input`
    uint64_t n_kmers;        // windows to process
    int64_t sym_base;        // symbol index of grid position 0 (= -phase)
    uint64_t* words;         // filter: num_shards * 4 words
    uint32_t shard_mask;     // (uint32_t)(num_shards - 1)
    uint8_t* out;            // query: one byte per window (null in bit-packed mode)
    uint32_t* out_bits;      // query, bit-packed mode: bit i % 32 of word i / 32
    uint64_t n_tiles;
    int* err;                // device error word (non-zero = failure code)
    // Ragged launches only.  Records sorted by offset and non-overlapping; a
    // window is processed only when its K bytes lie inside one record.
    const DevRange* ranges;
    uint64_t n_ranges;
    const uint32_t* tile_rec;      // per tile: first record whose end > tile start
    unsigned int* queue;           // work-queue counter, zero before the launch
    unsigned long long* counts;    // [0] valid windows, [1] positive windows
    // Optional per-record tallies (zeroed before the launch): valid and
    // positive windows of record r are added to rec_valid[r << rec_shift]
    // and rec_pos[r << rec_shift] (rec_shift 1 interleaves the two arrays).
    unsigned long long* rec_valid;
    unsigned long long* rec_pos;
    uint32_t rec_shift;
    GenericCfg gen;  // read by the generic kernels only
    // Ragged tile kernels: when set, input_bytes, n_kmers, n_tiles and
    // n_ranges are read from here at kernel start (n_tiles above is then the
    // host's upper bound, used only for the launch shape).
    const DevSizes* sizes;
};

// Device error codes written to TileParams::err.
enum : int {
    kDevErrNone = 0,
    kDevErrStageTimeout = 1,  // a bulk-copy wait ran out of its time bound
    kDevErrRecordRange = 2,   // sharded insert: a run record outside the rank's shards
};

// Function table for one compiled configuration <K,S,M,H> (k = s = m = h = 0
// for the generic table, whose kernels read TileParams::gen).
#ifndef __CUDACC_RTC__
// Kernels are launched with cudaLaunchKernel(fn, ...): a compiled kernel's
// host stub, or a cudaKernel_t of a kernel compiled at run time (jit).
struct KernelSet {
    int k, s, m, h;
    const void* insert_bytes;
    const void* query_bytes;
    const void* insert_dense;
    const void* query_dense;
    const void* insert_ragged;
    const void* query_ragged;
    // Dynamic shared memory of the insert and query kernels: the tile
    // kernels' flush ring and shard slots; none for the generic kernels.
    int smem_insert = kInsertSlotBytes;
    int smem_query = kQuerySlotBytes;
    bool jit = false;    // loaded from a run-time compiled library
    int jit_occupancy = 2;  // resident CTAs per SM assumed for run-time compiled sets
    int smem(bool query) const { return query ? smem_query : smem_insert; }
};

// Returns the kernel table for a configuration, or nullptr when it is not
// compiled into this library.
const KernelSet* find_kernels(int k, int s, int m, int h);
// The runtime-parameterised kernels (sbf_generic.cu).
const KernelSet* generic_kernels();

// Auxiliary kernels (sbf_kernels.cu).
cudaError_t launch_pack_dense(const uint8_t* seq, uint64_t num_symbols, uint64_t* words,
                              cudaStream_t stream);
// Ragged launches: tile_rec[t] = first record whose end exceeds the first
// input byte of tile t (n_ranges when none).
cudaError_t launch_tile_records(const DevRange* ranges, uint64_t n_ranges, int64_t sym_base,
                                uint64_t n_tiles, uint32_t* tile_rec, cudaStream_t stream);
// The same with the record and tile counts read from `sizes` on the device;
// `max_tiles` bounds the launch.
cudaError_t launch_tile_records_sized(const DevRange* ranges, const DevSizes* sizes,
                                      int64_t sym_base, uint64_t max_tiles, uint32_t* tile_rec,
                                      cudaStream_t stream);
cudaError_t launch_popcount(const uint64_t* words, uint64_t n_words, unsigned long long* out,
                            cudaStream_t stream);
// Kernels compiled at run time for a configuration that is not compiled into
// the library (sbf_jit.cpp): the tile kernels for DNA, the generic kernels
// with the configuration as constants for the other alphabets; nullptr when
// that is not possible.
const KernelSet* jit_kernels(int k, int s, int m, int h, int alphabet, int device);
// Launches one of a KernelSet's kernels.
cudaError_t launch_set_kernel(const KernelSet* ks, const void* fn, unsigned grid, bool query,
                              const TileParams& p, cudaStream_t stream);
#endif

}  // namespace sbf
