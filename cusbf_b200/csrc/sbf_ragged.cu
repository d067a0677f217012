// sbf_ragged.cu -- ragged batches: many records of uneven length through one
// persistent tile-kernel launch with a device work queue, a multi-stage host
// pipeline whose per-chunk device work can be replayed as a CUDA graph, and
// an autotuner with a persisted table.  No reference counterpart: the
// reference inserts a record batch by normalising it on the host (records
// joined with one 'N', include/cusbf/normalized_record_batch.hpp:235-276)
// and launching the plain kernel over the copy, or one launch per record
// (filter.cuh:179, :464).
//
// Records stay where they are.  The kernel marks, per staged tile, the
// first byte of every record and the bytes outside every record, and a
// window is valid only when its K bytes lie inside one record: exactly the
// windows of the reference's per-record insert/query.  Query output uses
// the batch's own layout: the hit of the window that starts at byte p of
// the batch is out[p], so record r's hits are out[offset_r, offset_r +
// bytes_r - K + 1) and windows that cross records read 0.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <sys/stat.h>
#include <string>
#include <vector>

#include "../../include/sbf_b200.h"
#include "sbf_expand.h"
#include "sbf_host.h"
#include "sbf_internal.h"
#include "sbf_ragged.h"

using namespace sbf;

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

static_assert(sizeof(DevRange) == sizeof(sbf_record_range), "record layout");

namespace sbf {

const void* tile_records_kernel_ptr();

constexpr int kMaxStages = 4;

// One stage of the host pipeline: pinned and device buffers of one chunk.
struct RaggedSlot {
    uint8_t* pin_seq = nullptr;
    size_t pin_seq_cap = 0;
    DevRange* pin_rng = nullptr;
    size_t pin_rng_cap = 0;
    uint8_t* d_seq = nullptr;
    size_t d_seq_cap = 0;
    DevRange* d_rng = nullptr;
    size_t d_rng_cap = 0;
    uint32_t* d_tile_rec = nullptr;
    size_t tile_cap = 0;
    uint8_t* d_out = nullptr;
    size_t out_cap = 0;
    // Bit-packed results of a byte-output query, expanded on the host once
    // downloaded: windows [pend_lo, pend_lo + pend_n) of the batch.
    uint32_t* pin_out = nullptr;
    size_t pin_out_cap = 0;
    uint64_t pend_lo = 0, pend_n = 0;
    bool pend = false;
    cudaEvent_t ev_copied = nullptr, ev_kernel = nullptr, ev_done = nullptr;
    bool busy = false;
    RaggedGraph graph[2];  // per operation (insert, query)
};

struct RaggedState {
    RaggedSlot slot[kMaxStages];
    cudaStream_t copy_stream = nullptr;  // chunk uploads
    cudaStream_t d2h_stream = nullptr;   // query result downloads
    // [0] work-queue counter; [2..3] (as u64) batch counts.
    unsigned int* d_ctl = nullptr;
    DevBuf direct_tile_rec;
};

template <class T>
static int grow_device(T*& p, size_t& cap, size_t bytes) {
    if (bytes <= cap) return SBF_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const size_t want = std::max<size_t>(bytes, 4096);
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(SBF_ERR_RESOURCE, "cannot allocate %zu bytes of ragged staging", want);
    }
    cap = want;
    return SBF_OK;
}

template <class T>
static int grow_pinned(T*& p, size_t& cap, size_t bytes) {
    if (bytes <= cap) return SBF_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    const size_t want = std::max<size_t>(bytes, 4096);
    cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&p), want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(SBF_ERR_RESOURCE, "cannot allocate %zu bytes of pinned staging", want);
    }
    cap = want;
    return SBF_OK;
}

static void release_slot(RaggedSlot& s) {
    if (s.pin_seq) cudaFreeHost(s.pin_seq);
    if (s.pin_rng) cudaFreeHost(s.pin_rng);
    if (s.pin_out) cudaFreeHost(s.pin_out);
    if (s.d_seq) cudaFree(s.d_seq);
    if (s.d_rng) cudaFree(s.d_rng);
    if (s.d_tile_rec) cudaFree(s.d_tile_rec);
    if (s.d_out) cudaFree(s.d_out);
    if (s.ev_copied) cudaEventDestroy(s.ev_copied);
    if (s.ev_kernel) cudaEventDestroy(s.ev_kernel);
    if (s.ev_done) cudaEventDestroy(s.ev_done);
    for (auto& g : s.graph) ragged_graph_release(g);
    s = RaggedSlot{};
}

void ragged_release(sbf_filter* f) {
    if (!f->ragged) return;
    RaggedState* r = f->ragged;
    for (auto& s : r->slot) release_slot(s);
    if (r->copy_stream) cudaStreamDestroy(r->copy_stream);
    if (r->d2h_stream) cudaStreamDestroy(r->d2h_stream);
    if (r->d_ctl) cudaFree(r->d_ctl);
    r->direct_tile_rec.release();
    delete r;
    f->ragged = nullptr;
}

static int ragged_state(sbf_filter* f, RaggedState** out) {
    if (!f->ragged) {
        auto* r = new RaggedState();
        f->ragged = r;
        cudaError_t e = cudaStreamCreateWithFlags(&r->copy_stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&r->d2h_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
        if ((e = cudaMalloc(&r->d_ctl, 64)) != cudaSuccess) return cuda_fail(e, "cudaMalloc(ctl)");
        if ((e = cudaMemset(r->d_ctl, 0, 64)) != cudaSuccess) return cuda_fail(e, "cudaMemset(ctl)");
        for (auto& s : r->slot) {
            if ((e = cudaEventCreateWithFlags(&s.ev_copied, cudaEventDisableTiming)) != cudaSuccess)
                return cuda_fail(e, "cudaEventCreate");
            if ((e = cudaEventCreateWithFlags(&s.ev_done, cudaEventDisableTiming)) != cudaSuccess)
                return cuda_fail(e, "cudaEventCreate");
            if ((e = cudaEventCreateWithFlags(&s.ev_kernel, cudaEventDisableTiming)) != cudaSuccess)
                return cuda_fail(e, "cudaEventCreate");
        }
    }
    *out = f->ragged;
    return SBF_OK;
}

static unsigned long long* ctl_counts(RaggedState* r) {
    return reinterpret_cast<unsigned long long*>(r->d_ctl + 2);
}

TileParams ragged_params(const sbf_filter* f, bool query, const uint8_t* d_seq,
                                uint64_t len, const DevRange* d_rng, uint64_t n,
                                const uint32_t* d_tile_rec, uint8_t* d_out, unsigned int* queue,
                                unsigned long long* counts, bool out_bits) {
    TileParams p{};
    p.input = d_seq;
    p.input_bytes = len;
    p.n_kmers = f->kmers_of_bytes(len);
    int64_t phase = 0;
    if (query && out_bits)
        phase = 0;  // strips start at multiples of 32 windows
    else if (query)
        phase = static_cast<int64_t>(reinterpret_cast<uintptr_t>(d_out) & 15u);
    else
        phase = static_cast<int64_t>(reinterpret_cast<uintptr_t>(d_seq) & 15u);
    p.sym_base = -phase;
    p.words = f->d_words;
    p.shard_mask = static_cast<uint32_t>(f->num_shards - 1);
    p.out = out_bits ? nullptr : d_out;
    p.out_bits = out_bits ? reinterpret_cast<uint32_t*>(d_out) : nullptr;
    p.n_tiles = (p.n_kmers + static_cast<uint64_t>(phase) + kTileKmers - 1) / kTileKmers;
    p.err = f->d_err;
    p.ranges = d_rng;
    p.n_ranges = n;
    p.tile_rec = d_tile_rec;
    p.queue = queue;
    p.counts = counts;
    p.gen = f->gen;
    return p;
}

static unsigned ragged_grid(const sbf_filter* f, bool query, uint64_t n_tiles, uint32_t ctas) {
    const int occ = f->occupancy[query ? 5 : 4];
    const uint64_t per_sm = ctas == 0 ? static_cast<uint64_t>(occ)
                                      : std::min<uint64_t>(ctas, static_cast<uint64_t>(occ));
    const uint64_t resident = static_cast<uint64_t>(f->sms) * std::max<uint64_t>(per_sm, 1);
    return static_cast<unsigned>(std::max<uint64_t>(std::min<uint64_t>(n_tiles, resident), 1));
}

int ragged_launch(sbf_filter* f, bool query, const TileParams& p, uint32_t ctas,
                         cudaStream_t st) {
    if (p.n_tiles == 0) return SBF_OK;
    SBF_CUDA(launch_tile_records(p.ranges, p.n_ranges, p.sym_base, p.n_tiles,
                                 const_cast<uint32_t*>(p.tile_rec), st));
    SBF_CUDA(cudaMemsetAsync(p.queue, 0, sizeof(unsigned int), st));
    const void* fn = query ? f->ks->query_ragged : f->ks->insert_ragged;
    SBF_CUDA(launch_set_kernel(f->ks, fn, ragged_grid(f, query, p.n_tiles, ctas), query, p, st));
    f->launches += 2;
    return SBF_OK;
}

// The graph is built on first use; later launches only update the two
// kernel nodes' parameters.
int ragged_graph_launch(sbf_filter* f, RaggedGraph& g, bool query, const TileParams& p,
                        uint32_t ctas, cudaStream_t st) {
    if (p.n_tiles == 0) return SBF_OK;
    // Graph kernel nodes take compiled kernels; run-time compiled ones are
    // launched on the stream.
    if (f->ks->jit) return ragged_launch(f, query, p, ctas, st);
    const DevRange* a_rng = p.ranges;
    uint64_t a_n = p.n_ranges;
    int64_t a_base = p.sym_base;
    uint64_t a_tiles = p.n_tiles;
    uint32_t* a_rec = const_cast<uint32_t*>(p.tile_rec);
    void* rec_args[] = {&a_rng, &a_n, &a_base, &a_tiles, &a_rec};
    TileParams tp = p;
    void* tile_args[] = {&tp};
    cudaKernelNodeParams rk{};
    rk.func = const_cast<void*>(tile_records_kernel_ptr());
    rk.gridDim = dim3(static_cast<unsigned>((p.n_tiles + 255) / 256));
    rk.blockDim = dim3(256);
    rk.kernelParams = rec_args;
    cudaKernelNodeParams tk{};
    tk.func = const_cast<void*>(query ? f->ks->query_ragged : f->ks->insert_ragged);
    tk.gridDim = dim3(ragged_grid(f, query, p.n_tiles, ctas));
    tk.blockDim = dim3(kThreads);
    tk.sharedMemBytes = f->ks->smem(query);
    tk.kernelParams = tile_args;
    if (!g.exec) {
        SBF_CUDA(cudaGraphCreate(&g.graph, 0));
        SBF_CUDA(cudaGraphAddKernelNode(&g.n_rec, g.graph, nullptr, 0, &rk));
        cudaMemsetParams ms{};
        ms.dst = p.queue;
        ms.value = 0;
        ms.elementSize = sizeof(unsigned int);
        ms.width = 1;
        ms.height = 1;
        cudaGraphNode_t n_ms;
        SBF_CUDA(cudaGraphAddMemsetNode(&n_ms, g.graph, &g.n_rec, 1, &ms));
        SBF_CUDA(cudaGraphAddKernelNode(&g.n_tile, g.graph, &n_ms, 1, &tk));
        SBF_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
    } else {
        SBF_CUDA(cudaGraphExecKernelNodeSetParams(g.exec, g.n_rec, &rk));
        SBF_CUDA(cudaGraphExecKernelNodeSetParams(g.exec, g.n_tile, &tk));
    }
    SBF_CUDA(cudaGraphLaunch(g.exec, st));
    f->launches += 2;
    return SBF_OK;
}

void ragged_graph_release(RaggedGraph& g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g = RaggedGraph{};
}

// ---------------------------------------------------------------------------
// Tuning table
// ---------------------------------------------------------------------------

struct TuneKey {
    int op, k, s, m, h, len_bucket, rec_bucket;
};

static int log2_bucket(double v) { return v < 1 ? 0 : static_cast<int>(std::floor(std::log2(v))); }

static TuneKey tune_key(const sbf_filter* f, bool query, uint64_t len, uint64_t n) {
    return TuneKey{query ? 1 : 0,
                   static_cast<int>(f->k),
                   static_cast<int>(f->s),
                   static_cast<int>(f->m),
                   static_cast<int>(f->h),
                   log2_bucket(static_cast<double>(len)),
                   log2_bucket(n ? static_cast<double>(len) / static_cast<double>(n) : 0.0)};
}

static std::string tune_table_path() {
    if (const char* p = std::getenv("SBF_TUNE_TABLE")) return p;
    const char* home = std::getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/cusbf_b200/ragged_tuning.tsv";
}

static std::mutex g_tune_mutex;

static bool tune_lookup(const TuneKey& key, sbf_ragged_tuning* out) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    FILE* fp = std::fopen(tune_table_path().c_str(), "r");
    if (!fp) return false;
    char line[256];
    bool found = false;
    while (std::fgets(line, sizeof line, fp)) {
        TuneKey k{};
        unsigned long long chunk = 0;
        unsigned stages = 0, ctas = 0, graph = 0;
        if (std::sscanf(line, "%d %d %d %d %d %d %d %llu %u %u %u", &k.op, &k.k, &k.s, &k.m, &k.h,
                        &k.len_bucket, &k.rec_bucket, &chunk, &stages, &ctas, &graph) != 11)
            continue;
        if (std::memcmp(&k, &key, sizeof k) == 0) {  // the last matching line wins
            out->chunk_bytes = chunk;
            out->stages = stages;
            out->ctas_per_sm = ctas;
            out->use_graph = graph;
            found = true;
        }
    }
    std::fclose(fp);
    return found;
}

static void tune_store(const TuneKey& key, const sbf_ragged_tuning& t, double ms) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    const std::string path = tune_table_path();
    // Create the table's directory chain; existing directories are kept.
    for (size_t i = 1; i < path.size(); ++i)
        if (path[i] == '/') (void)mkdir(path.substr(0, i).c_str(), 0755);
    FILE* fp = std::fopen(path.c_str(), "a");
    if (!fp) return;
    std::fprintf(fp, "%d %d %d %d %d %d %d %llu %u %u %u %.4f\n", key.op, key.k, key.s, key.m,
                 key.h, key.len_bucket, key.rec_bucket,
                 static_cast<unsigned long long>(t.chunk_bytes), t.stages, t.ctas_per_sm,
                 t.use_graph, ms);
    std::fclose(fp);
}

// Defaults when no tuning-table entry matches: queries stage larger chunks,
// three in flight (the shape the autotuner picks for read batches; their
// uploads are the larger stream), inserts 64 MiB chunks, two in flight.
static sbf_ragged_tuning default_tuning(bool query = false) {
    sbf_ragged_tuning t{};
    t.chunk_bytes = query ? uint64_t{256} << 20 : uint64_t{64} << 20;
    t.stages = query ? 3 : 2;
    t.ctas_per_sm = 0;
    t.use_graph = 0;
    return t;
}

// Zero fields take the operation's defaults.
static int check_tuning(sbf_ragged_tuning& t, bool query) {
    if (t.chunk_bytes == 0) t.chunk_bytes = default_tuning(query).chunk_bytes;
    if (t.chunk_bytes < 4096)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "ragged chunk_bytes must be at least 4096");
    if (t.stages == 0) t.stages = default_tuning(query).stages;
    if (t.stages < 1 || t.stages > kMaxStages)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "ragged stages must be 1..%d", kMaxStages);
    return SBF_OK;
}

// ---------------------------------------------------------------------------
// Host pipeline
// ---------------------------------------------------------------------------

// Clips chunk-overlapping records to the chunk's bytes [b_lo, b_hi) and
// rebases them to the chunk, in place.  Pieces shorter than K hold no window;
// the windows that cross one span a record start or bytes outside every
// record either way, so they stay invalid.
__global__ void clip_ranges_kernel(DevRange* r, uint64_t n, uint64_t b_lo, uint64_t b_hi) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const DevRange x = r[i];
        const uint64_t a = x.offset > b_lo ? x.offset : b_lo;
        const uint64_t end = x.offset + x.bytes;
        const uint64_t e = end < b_hi ? end : b_hi;
        r[i] = DevRange{a - b_lo, e > a ? e - a : 0};
    }
}

// Windows [0, W) of the batch are cut into chunks of `cw` windows; chunk c
// stages bytes [c*cw, c*cw + cw + K - 1) and the records that overlap them,
// copied as given (one memcpy of the slice) and clipped on the GPU.
// With h_bits, query results are bit-packed (window i -> bit i % 32 of word
// i / 32) and chunks hold a multiple of 32 windows, so each chunk's result
// words start on a word boundary.
static int ragged_pipeline(sbf_filter* f, bool query, const char* h_seq, uint64_t len,
                           const sbf_record_range* ranges, uint64_t n, sbf_ragged_tuning t,
                           cudaStream_t st, uint8_t* h_out, unsigned long long counts[2],
                           uint32_t* h_bits = nullptr) {
    counts[0] = counts[1] = 0;
    const bool bits = h_bits != nullptr;
    const uint64_t K = f->k;
    const uint64_t W = f->kmers_of(len);
    if (W == 0 || n == 0) {
        if (query && W) std::memset(bits ? reinterpret_cast<uint8_t*>(h_bits) : h_out, 0,
                                    bits ? (W + 31) / 32 * 4 : W);
        return SBF_OK;
    }
    // Byte results come down one bit per window and are expanded by host
    // threads (kbits: the kernel writes bit-packed results).
    ExpandPool* pool = query && !bits ? host_expand_pool(f) : nullptr;
    const bool kbits = bits || pool != nullptr;
    auto out_bytes = [&](uint64_t windows) { return kbits ? (windows + 31) / 32 * 4 : windows; };
    RaggedState* r = nullptr;
    SBF_TRY(ragged_state(f, &r));
    SBF_TRY(check_tuning(t, query));
    uint64_t cw = std::max<uint64_t>(t.chunk_bytes > K ? t.chunk_bytes - (K - 1) : 1, 1024);
    if (kbits) cw = std::max<uint64_t>(cw / 32 * 32, 1024);
    const uint64_t n_chunks = (W + cw - 1) / cw;
    const uint64_t max_bytes = cw + K - 1;
    const uint64_t max_pieces = max_bytes / K + 2;
    const bool pinned_in = is_pinned(h_seq);
    const bool pinned_rng = is_pinned(ranges);  // slices upload without a host copy
    unsigned long long* d_counts = ctl_counts(r);
    SBF_CUDA(cudaMemsetAsync(d_counts, 0, 2 * sizeof(unsigned long long), st));
    const uint32_t S = t.stages;
    for (uint32_t i = 0; i < S; ++i) {
        RaggedSlot& s = r->slot[i];
        if (!pinned_in) SBF_TRY(grow_pinned(s.pin_seq, s.pin_seq_cap, max_bytes + 16));
        SBF_TRY(grow_pinned(s.pin_rng, s.pin_rng_cap, max_pieces * sizeof(DevRange)));
        SBF_TRY(grow_device(s.d_seq, s.d_seq_cap, max_bytes + 16));
        SBF_TRY(grow_device(s.d_rng, s.d_rng_cap, max_pieces * sizeof(DevRange)));
        SBF_TRY(grow_device(s.d_tile_rec, s.tile_cap, ((cw + 16) / kTileKmers + 2) * 4));
        if (query) SBF_TRY(grow_device(s.d_out, s.out_cap, out_bytes(cw) + 16));
        if (pool) SBF_TRY(grow_pinned(s.pin_out, s.pin_out_cap, out_bytes(cw) + 16));
        s.busy = false;
        s.pend = false;
    }
    // The copy stream starts after work already queued on `st`.
    cudaEvent_t ev_start = r->slot[0].ev_done;
    SBF_CUDA(cudaEventRecord(ev_start, st));
    SBF_CUDA(cudaStreamWaitEvent(r->copy_stream, ev_start, 0));
    SBF_CUDA(cudaStreamWaitEvent(r->d2h_stream, ev_start, 0));
    uint64_t rec = 0;      // first record whose end exceeds the chunk's first byte
    uint64_t rec_end = 0;  // first record that starts at or after the chunk's end
    for (uint64_t c = 0; c < n_chunks; ++c) {
        RaggedSlot& s = r->slot[c % S];
        if (s.busy) SBF_CUDA(cudaEventSynchronize(s.ev_done));
        if (s.pend) {
            pool->run(s.pin_out, h_out + s.pend_lo, s.pend_n);
            s.pend = false;
        }
        const uint64_t w_lo = c * cw;
        const uint64_t w_hi = std::min<uint64_t>(W, w_lo + cw);
        const uint64_t b_lo = w_lo, b_hi = w_hi + K - 1;
        // Validated records are ordered and non-overlapping, so both their
        // starts and their ends are non-decreasing: binary searches find the
        // chunk's records without touching the ones in between.
        rec = static_cast<uint64_t>(
            std::partition_point(ranges + rec, ranges + n,
                                 [b_lo](const sbf_record_range& x) {
                                     return x.sequence_offset + x.sequence_bytes <= b_lo;
                                 }) -
            ranges);
        rec_end = static_cast<uint64_t>(
            std::partition_point(ranges + std::max(rec_end, rec), ranges + n,
                                 [b_hi](const sbf_record_range& x) {
                                     return x.sequence_offset < b_hi;
                                 }) -
            ranges);
        const uint64_t np = rec_end - rec;
        if (np * sizeof(DevRange) > s.pin_rng_cap || np * sizeof(DevRange) > s.d_rng_cap) {
            // Many records shorter than K in one chunk: grow with headroom.
            SBF_TRY(grow_pinned(s.pin_rng, s.pin_rng_cap, 2 * np * sizeof(DevRange)));
            SBF_TRY(grow_device(s.d_rng, s.d_rng_cap, 2 * np * sizeof(DevRange)));
        }
        const void* rng_src = ranges + rec;
        if (np && !pinned_rng) {
            std::memcpy(s.pin_rng, ranges + rec, np * sizeof(DevRange));
            rng_src = s.pin_rng;
        }
        const uint8_t* src = reinterpret_cast<const uint8_t*>(h_seq) + b_lo;
        if (!pinned_in) {
            std::memcpy(s.pin_seq, src, b_hi - b_lo);
            src = s.pin_seq;
        }
        SBF_CUDA(cudaMemcpyAsync(s.d_seq, src, b_hi - b_lo, cudaMemcpyHostToDevice,
                                 r->copy_stream));
        if (np)
            SBF_CUDA(cudaMemcpyAsync(s.d_rng, rng_src, np * sizeof(DevRange),
                                     cudaMemcpyHostToDevice, r->copy_stream));
        SBF_CUDA(cudaEventRecord(s.ev_copied, r->copy_stream));
        SBF_CUDA(cudaStreamWaitEvent(st, s.ev_copied, 0));
        if (np) {
            const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((np + 255) / 256, 1024));
            clip_ranges_kernel<<<blocks, 256, 0, st>>>(s.d_rng, np, b_lo, b_hi);
            SBF_CUDA(cudaGetLastError());
            const TileParams p = ragged_params(f, query, s.d_seq, b_hi - b_lo, s.d_rng, np,
                                               s.d_tile_rec, s.d_out, r->d_ctl, d_counts, kbits);
            if (t.use_graph)
                SBF_TRY(ragged_graph_launch(f, s.graph[query ? 1 : 0], query, p, t.ctas_per_sm,
                                            st));
            else
                SBF_TRY(ragged_launch(f, query, p, t.ctas_per_sm, st));
        } else if (query) {
            SBF_CUDA(cudaMemsetAsync(s.d_out, 0, out_bytes(w_hi - w_lo), st));
        }
        // Downloads run on their own stream so the next chunk's kernel does
        // not queue behind this chunk's download.  The host waits for
        // ev_done before it refills this slot, so no stream waits on a later
        // chunk's work.
        if (query) {
            SBF_CUDA(cudaEventRecord(s.ev_kernel, st));
            SBF_CUDA(cudaStreamWaitEvent(r->d2h_stream, s.ev_kernel, 0));
            void* dst = bits   ? static_cast<void*>(h_bits + w_lo / 32)
                        : pool ? static_cast<void*>(s.pin_out)
                               : static_cast<void*>(h_out + w_lo);
            SBF_CUDA(cudaMemcpyAsync(dst, s.d_out, out_bytes(w_hi - w_lo), cudaMemcpyDeviceToHost,
                                     r->d2h_stream));
            if (pool) {
                s.pend = true;
                s.pend_lo = w_lo;
                s.pend_n = w_hi - w_lo;
            }
            SBF_CUDA(cudaEventRecord(s.ev_done, r->d2h_stream));
        } else {
            SBF_CUDA(cudaEventRecord(s.ev_done, st));
        }
        s.busy = true;
    }
    if (pool) {
        // The last chunks, each as soon as its download is done.
        const uint64_t first = n_chunks > S ? n_chunks - S : 0;
        for (uint64_t c = first; c < n_chunks; ++c) {
            RaggedSlot& s = r->slot[c % S];
            if (!s.pend) continue;
            SBF_CUDA(cudaEventSynchronize(s.ev_done));
            pool->run(s.pin_out, h_out + s.pend_lo, s.pend_n);
            s.pend = false;
        }
    }
    SBF_CUDA(cudaEventRecord(r->slot[0].ev_kernel, r->d2h_stream));
    SBF_CUDA(cudaStreamWaitEvent(st, r->slot[0].ev_kernel, 0));
    unsigned long long h_counts[2] = {0, 0};
    SBF_CUDA(cudaMemcpyAsync(h_counts, d_counts, sizeof h_counts, cudaMemcpyDeviceToHost, st));
    SBF_CUDA(cudaStreamSynchronize(st));
    for (uint32_t i = 0; i < S; ++i) r->slot[i].busy = false;
    SBF_TRY(f->check_device_error(st));
    counts[0] = h_counts[0];
    counts[1] = h_counts[1];
    return SBF_OK;
}

static int resolve_tuning(const sbf_filter* f, bool query, uint64_t len, uint64_t n,
                          const sbf_ragged_tuning* given, sbf_ragged_tuning* out) {
    if (given) {
        *out = *given;
    } else if (!tune_lookup(tune_key(f, query, len, n), out)) {
        *out = default_tuning(query);
    }
    return check_tuning(*out, query);
}

}  // namespace sbf

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

static inline cudaStream_t S_(sbf_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

static int ragged_async(sbf_filter_t* f, bool query, const char* d_seq, uint64_t len,
                        const sbf_record_range* d_ranges, uint64_t n, uint8_t* d_out,
                        uint64_t out_len, uint64_t* d_counts, sbf_stream_t stream,
                        uint64_t* d_rec_valid = nullptr, uint64_t* d_rec_pos = nullptr) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    if (n && !d_ranges) return set_error(SBF_ERR_INVALID_ARGUMENT, "ranges pointer is null");
    if (n > 0xFFFFFFFFull) return set_error(SBF_ERR_INVALID_ARGUMENT, "too many records");
    const bool tally = d_rec_valid != nullptr;
    if (tally && n && !d_rec_pos)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "per-record count arrays are null");
    cudaStream_t st = S_(stream);
    if (tally && n) {
        SBF_CUDA(cudaMemsetAsync(d_rec_valid, 0, n * sizeof(uint64_t), st));
        SBF_CUDA(cudaMemsetAsync(d_rec_pos, 0, n * sizeof(uint64_t), st));
    }
    const uint64_t W = f->kmers_of_bytes(len);
    if (W == 0) return SBF_OK;
    if (!d_seq) return set_error(SBF_ERR_INVALID_ARGUMENT, "sequence pointer is null");
    // With per-record counts the hit bytes are optional.
    if (query && (tally ? (d_out && out_len < W) : (!d_out || out_len < W)))
        return set_error(SBF_ERR_INVALID_ARGUMENT, "ragged query output span is too small");
    RaggedState* r = nullptr;
    SBF_TRY(ragged_state(f, &r));
    if (n == 0) {
        if (query && d_out) SBF_CUDA(cudaMemsetAsync(d_out, 0, W, st));
        return SBF_OK;
    }
    TileParams p = ragged_params(f, query, reinterpret_cast<const uint8_t*>(d_seq), len,
                                 reinterpret_cast<const DevRange*>(d_ranges), n, nullptr, d_out,
                                 r->d_ctl,
                                 d_counts ? reinterpret_cast<unsigned long long*>(d_counts)
                                          : ctl_counts(r));
    p.rec_valid = reinterpret_cast<unsigned long long*>(d_rec_valid);
    p.rec_pos = reinterpret_cast<unsigned long long*>(d_rec_pos);
    SBF_TRY(r->direct_tile_rec.ensure(p.n_tiles * 4 + 64));
    p.tile_rec = static_cast<const uint32_t*>(r->direct_tile_rec.ptr);
    return ragged_launch(f, query, p, 0, st);
}

extern "C" int sbf_ragged_insert_async(sbf_filter_t* f, const char* d_seq, uint64_t len,
                                       const sbf_record_range* d_ranges, uint64_t n,
                                       uint64_t* d_counts, sbf_stream_t stream) {
    return ragged_async(f, false, d_seq, len, d_ranges, n, nullptr, 0, d_counts, stream);
}

extern "C" int sbf_ragged_contains_async(const sbf_filter_t* f, const char* d_seq, uint64_t len,
                                         const sbf_record_range* d_ranges, uint64_t n,
                                         uint8_t* d_out, uint64_t out_len, uint64_t* d_counts,
                                         sbf_stream_t stream) {
    return ragged_async(const_cast<sbf_filter*>(f), true, d_seq, len, d_ranges, n, d_out, out_len,
                        d_counts, stream);
}

extern "C" int sbf_ragged_contains_counts_async(const sbf_filter_t* f, const char* d_seq,
                                                uint64_t len, const sbf_record_range* d_ranges,
                                                uint64_t n, uint8_t* d_out, uint64_t out_len,
                                                uint64_t* d_record_valid,
                                                uint64_t* d_record_positive, uint64_t* d_counts,
                                                sbf_stream_t stream) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    if (n == 0) {
        // No records: nothing to count; a given output span reads all 0.
        return d_out ? ragged_async(const_cast<sbf_filter*>(f), true, d_seq, len, d_ranges, 0,
                                    d_out, out_len, d_counts, stream)
                     : SBF_OK;
    }
    if (!d_record_valid || !d_record_positive)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "per-record count arrays are null");
    return ragged_async(const_cast<sbf_filter*>(f), true, d_seq, len, d_ranges, n, d_out, out_len,
                        d_counts, stream, d_record_valid, d_record_positive);
}

extern "C" int sbf_ragged_insert(sbf_filter_t* f, const char* h_seq, uint64_t len,
                                 const sbf_record_range* ranges, uint64_t n,
                                 const sbf_ragged_tuning* tuning, sbf_stream_t stream,
                                 sbf_insert_report* report) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    SBF_TRY(f->require_byte_symbols("the ragged host pipeline"));
    if (n && (!ranges || !h_seq)) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    uint64_t bases = 0;
    SBF_TRY(validate_ranges(len, ranges, n, &bases));
    sbf_ragged_tuning t{};
    SBF_TRY(resolve_tuning(f, false, len, n, tuning, &t));
    unsigned long long counts[2];
    SBF_TRY(ragged_pipeline(f, false, h_seq, len, ranges, n, t, S_(stream), nullptr, counts));
    if (report) {
        report->records_indexed = n;
        report->indexed_bases = bases;
        report->inserted_kmers = counts[0];
    }
    return SBF_OK;
}

extern "C" int sbf_ragged_query(const sbf_filter_t* cf, const char* h_seq, uint64_t len,
                                const sbf_record_range* ranges, uint64_t n, uint8_t* h_out,
                                uint64_t out_len, const sbf_ragged_tuning* tuning,
                                sbf_stream_t stream, sbf_query_report* report) {
    auto* f = const_cast<sbf_filter*>(cf);
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    SBF_TRY(f->require_byte_symbols("the ragged host pipeline"));
    if (n && (!ranges || !h_seq)) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    uint64_t bases = 0;
    SBF_TRY(validate_ranges(len, ranges, n, &bases));
    const uint64_t W = f->kmers_of(len);
    if (W && (!h_out || out_len < W))
        return set_error(SBF_ERR_INVALID_ARGUMENT, "ragged query output span is too small");
    sbf_ragged_tuning t{};
    SBF_TRY(resolve_tuning(f, true, len, n, tuning, &t));
    unsigned long long counts[2];
    SBF_TRY(ragged_pipeline(f, true, h_seq, len, ranges, n, t, S_(stream), h_out, counts));
    if (report) {
        report->records_queried = n;
        report->queried_bases = bases;
        report->queried_kmers = counts[0];
        report->positive_kmers = counts[1];
    }
    return SBF_OK;
}

extern "C" int sbf_ragged_query_bits(const sbf_filter_t* cf, const char* h_seq, uint64_t len,
                                     const sbf_record_range* ranges, uint64_t n, uint32_t* h_bits,
                                     uint64_t n_words, const sbf_ragged_tuning* tuning,
                                     sbf_stream_t stream, sbf_query_report* report) {
    auto* f = const_cast<sbf_filter*>(cf);
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    SBF_TRY(f->require_byte_symbols("the ragged host pipeline"));
    if (n && (!ranges || !h_seq)) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    uint64_t bases = 0;
    SBF_TRY(validate_ranges(len, ranges, n, &bases));
    const uint64_t W = f->kmers_of(len);
    if (W && (!h_bits || n_words < (W + 31) / 32))
        return set_error(SBF_ERR_INVALID_ARGUMENT, "ragged query bit output span is too small");
    sbf_ragged_tuning t{};
    SBF_TRY(resolve_tuning(f, true, len, n, tuning, &t));
    unsigned long long counts[2];
    SBF_TRY(ragged_pipeline(f, true, h_seq, len, ranges, n, t, S_(stream), nullptr, counts,
                            h_bits));
    if (report) {
        report->records_queried = n;
        report->queried_bases = bases;
        report->queried_kmers = counts[0];
        report->positive_kmers = counts[1];
    }
    return SBF_OK;
}

extern "C" int sbf_ragged_tuning_lookup(const sbf_filter_t* f, int query, uint64_t len,
                                        uint64_t n, sbf_ragged_tuning* out) {
    if (!f || !out) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    if (tune_lookup(tune_key(f, query != 0, len, n), out)) return SBF_OK;
    *out = default_tuning(query != 0);
    return set_error(SBF_ERR_INVALID_ARGUMENT, "no tuned entry for this shape (defaults returned)");
}

// Times candidate tunings on a prefix of the batch (records clipped to
// `sample_bytes`) through the host pipeline, keeps the fastest and appends
// it to the tuning table.  Inserting the prefix is idempotent for a batch
// that is then inserted in full.
extern "C" int sbf_ragged_autotune(sbf_filter_t* f, int query, const char* h_seq, uint64_t len,
                                   const sbf_record_range* ranges, uint64_t n,
                                   uint64_t sample_bytes, sbf_stream_t stream,
                                   sbf_ragged_tuning* chosen) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    SBF_TRY(f->require_byte_symbols("the ragged host pipeline"));
    if (n && (!ranges || !h_seq)) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    SBF_TRY(validate_ranges(len, ranges, n));
    // Four of the largest candidate chunks, so the sample shows pipelining.
    if (sample_bytes == 0) sample_bytes = uint64_t{1} << 30;
    const uint64_t sl = std::min<uint64_t>(len, sample_bytes);
    uint64_t sn = 0;
    while (sn < n && ranges[sn].sequence_offset < sl) ++sn;
    std::vector<sbf_record_range> sr(ranges, ranges + sn);
    if (sn && sr[sn - 1].sequence_offset + sr[sn - 1].sequence_bytes > sl)
        sr[sn - 1].sequence_bytes = sl - sr[sn - 1].sequence_offset;
    // Pinned result buffer, as a streaming caller would use: downloads into
    // pageable memory would slow every candidate and skew the choice.
    PinnedBuf out;
    struct Release {
        PinnedBuf& b;
        ~Release() { b.release(); }
    } release_out{out};
    SBF_TRY(out.ensure(query ? std::max<uint64_t>(f->kmers_of(sl), 1) : 1));
    const uint64_t chunks[] = {uint64_t{16} << 20, uint64_t{64} << 20, uint64_t{256} << 20};
    const uint32_t stage_opts[] = {2, 3};
    const uint32_t graph_opts[] = {0, 1};
    sbf_ragged_tuning best = default_tuning();
    double best_ms = 1e300;
    auto time_one = [&](const sbf_ragged_tuning& t, double* ms_out) -> int {
        unsigned long long counts[2];
        double ms = 1e300;
        for (int rep = 0; rep < 2; ++rep) {  // the first run warms buffers and graphs
            const auto t0 = std::chrono::steady_clock::now();
            SBF_TRY(ragged_pipeline(f, query != 0, h_seq, sl, sr.data(), sn, t, S_(stream),
                                    static_cast<uint8_t*>(out.p), counts));
            const auto t1 = std::chrono::steady_clock::now();
            ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        }
        *ms_out = ms;
        return SBF_OK;
    };
    // Chunk length x staging depth x graph replay, at the occupancy limit.
    for (uint64_t cb : chunks) {
        if (cb > 2 * sl && cb != chunks[0]) continue;  // larger chunks only repeat the smaller
        for (uint32_t stg : stage_opts)
            for (uint32_t gr : graph_opts) {
                const sbf_ragged_tuning t{cb, stg, 0, gr};
                double ms;
                SBF_TRY(time_one(t, &ms));
                if (ms < best_ms) {
                    best_ms = ms;
                    best = t;
                }
            }
    }
    // Warps per SM for the winner: one CTA (8 warps) instead of the
    // occupancy limit, which leaves SM room for concurrent work.
    {
        sbf_ragged_tuning t = best;
        t.ctas_per_sm = 1;
        double ms;
        SBF_TRY(time_one(t, &ms));
        if (ms < best_ms) {
            best_ms = ms;
            best = t;
        }
    }
    tune_store(tune_key(f, query != 0, len, n), best, best_ms);
    if (chosen) *chosen = best;
    return SBF_OK;
}
