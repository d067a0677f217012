// sbf_shard.cu -- device steps of the sharded multi-rank insert: run records
// are emitted instead of ORed into a filter (sbf_emit_runs_async), and the
// records a rank owns are ORed into its shard range (sbf_apply_runs_async).
// The exchange between the two runs on the host side (cusbf_b200/sharded.py,
// torch.distributed all-to-all over NCCL).
//
// Reference path replaced, when ranks split one input: the single-GPU insert
// include/cusbf/detail/kernels.cuh:107-172, 214-242 of tdortman/cuSBF, which
// ORs every run's word masks into its shard (filter_ref.cuh:94-108).  OR is
// order-independent, so emitting the same runs and ORing them anywhere later
// gives the same filter words.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/sbf_b200.h"
#include "sbf_host.h"
#include "sbf_internal.h"
#include "sbf_tile.cuh"

namespace sbf {
namespace {

// Per-CTA record staging in dynamic shared memory: kLogRecords records of a
// 4-byte shard id and four 8-byte masks.  A tile of 8192 windows emits about
// 1000 runs of uniform DNA; a tile with more than kLogRecords runs appends the
// excess to the global log one record at a time.
constexpr int kLogRecords = 1536;
constexpr int kEmitSmem = kLogRecords * (32 + 4);

struct RunLog {
    uint32_t* shards;   // [capacity]
    uint64_t* masks;    // [capacity][4]
    uint64_t capacity;
    unsigned long long* count;  // [0] records emitted (may exceed capacity), [1] valid windows
};

__device__ __forceinline__ void log_put(const RunLog& log, uint64_t at, uint32_t shard,
                                        const uint64_t* m) {
    if (at >= log.capacity) return;  // counted, not stored: the caller retries larger
    log.shards[at] = shard;
    *reinterpret_cast<ulonglong2*>(log.masks + 4 * at) = make_ulonglong2(m[0], m[1]);
    *reinterpret_cast<ulonglong2*>(log.masks + 4 * at + 2) = make_ulonglong2(m[2], m[3]);
}

// The insert tile path (plain loads for staging) with each super-k-mer run
// appended to the CTA's shared-memory log; at the end of every tile the CTA
// reserves a contiguous range of the global log with one atomic and copies
// its records there.
template <class C>
__global__ void __launch_bounds__(kThreads, 2) emit_kernel(TileParams p, RunLog log) {
    __shared__ alignas(16) uint8_t stage[kStageBytes];
    __shared__ uint32_t code[kCodeWords + 4];
    __shared__ uint32_t inval[kCodeWords + 4];
    __shared__ unsigned int cta_n;
    __shared__ unsigned long long cta_base;
    __shared__ uint64_t onehot[64];
    extern __shared__ __align__(16) uint64_t dyn[];
    uint64_t* s_masks = dyn;                                          // [kLogRecords][4]
    uint32_t* s_shards = reinterpret_cast<uint32_t*>(dyn + 4 * kLogRecords);  // [kLogRecords]
    const int tid = threadIdx.x;
    if (tid == 0) cta_n = 0;
    onehot_init(onehot);  // published by the barrier at the top of the tile loop
    unsigned long long n_valid = 0;
    for (uint64_t tile = blockIdx.x; tile < p.n_tiles; tile += gridDim.x) {
        TileGeom g = tile_geom<false>(p, tile);
        g.hi = g.lo;  // no bulk copy: every readable byte by plain loads
        __syncthreads();
        fill_ragged<false>(p, g, stage);
        __syncthreads();
        for (int q = tid; q < kCodeWords; q += kThreads) {
            uint32_t cw, iv;
            encode_word<false>(g, stage, q, cw, iv);
            code[q] = cw;
            inval[q] = iv;
        }
        __syncthreads();
        uint32_t c[kStripWords], iv[kStripWords];
#pragma unroll
        for (int q = 0; q < kStripWords; ++q) {
            c[q] = code[tid * (kStrip / 16) + q];
            iv[q] = inval[tid * (kStrip / 16) + q];
        }
        const int64_t first_kmer = g.s0 + static_cast<int64_t>(tid) * kStrip;
        const uint32_t vmask = strip_valid<C>(iv, first_kmer, p.n_kmers);
        n_valid += __popc(vmask);
        if (vmask)
            insert_strip<C>(c, vmask, p.shard_mask, onehot, [&](uint32_t end, uint32_t shard,
                                                        const uint64_t* acc) {
                if (!end) return;
                const unsigned int i = atomicAdd(&cta_n, 1u);
                if (i < static_cast<unsigned int>(kLogRecords)) {
                    s_shards[i] = shard;
                    *reinterpret_cast<ulonglong2*>(s_masks + 4 * i) = make_ulonglong2(acc[0], acc[1]);
                    *reinterpret_cast<ulonglong2*>(s_masks + 4 * i + 2) =
                        make_ulonglong2(acc[2], acc[3]);
                } else {
                    log_put(log, atomicAdd(log.count, 1ull), shard, acc);
                }
            });
        __syncthreads();
        const unsigned int n = min(cta_n, static_cast<unsigned int>(kLogRecords));
        if (tid == 0) cta_base = n ? atomicAdd(log.count, static_cast<unsigned long long>(n)) : 0;
        __syncthreads();
        for (unsigned int i = tid; i < n; i += kThreads) log_put(log, cta_base + i, s_shards[i], s_masks + 4 * i);
        __syncthreads();
        if (tid == 0) cta_n = 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n_valid += __shfl_down_sync(0xFFFFFFFFu, n_valid, o);
    if ((tid & 31) == 0 && n_valid) atomicAdd(log.count + 1, n_valid);
}

// ORs records whose shards lie in [lo, hi) into the filter, each with one
// 32-byte bulk OR-reduction from the thread's shared-memory ring (one L2
// operation per record, as the insert kernel flushes its runs); a record
// outside the range sets the error word (it was routed to the wrong rank).
__global__ void __launch_bounds__(kThreads) apply_runs_kernel(const uint32_t* shards,
                                                              const uint64_t* masks, uint64_t n,
                                                              uint64_t* words, uint64_t lo,
                                                              uint64_t hi, int* err) {
    extern __shared__ __align__(16) uint64_t ring_mem[];
    FlushRing ring{ring_mem + 4 * threadIdx.x, 0u};
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t sh = shards[i];
        if (sh < lo || sh >= hi) {
            atomicExch(err, kDevErrRecordRange);
            continue;
        }
        const ulonglong2 a = *reinterpret_cast<const ulonglong2*>(masks + 4 * i);
        const ulonglong2 b = *reinterpret_cast<const ulonglong2*>(masks + 4 * i + 2);
        const uint64_t m[4] = {a.x, a.y, b.x, b.y};
        flush_run(words, static_cast<uint32_t>(sh), m, ring);
    }
    flush_ring_drain();
}

using EmitFn = void (*)(TileParams, RunLog);

struct EmitSet {
    int k, s, m, h;
    EmitFn fn;
};

template <int K, int S, int M, int H>
constexpr EmitSet emit_set() {
    return EmitSet{K, S, M, H, &emit_kernel<Cfg<K, S, M, H>>};
}

// The configurations whose tile kernels are compiled into the library.
const EmitSet kEmitSets[] = {
    emit_set<31, 28, 16, 4>(),  emit_set<31, 30, 16, 4>(), emit_set<31, 31, 16, 4>(),
    emit_set<31, 28, 16, 8>(),  emit_set<31, 28, 16, 16>(), emit_set<21, 19, 11, 4>(),
    emit_set<5, 4, 3, 4>(),     emit_set<3, 2, 2, 4>(),     emit_set<31, 28, 21, 4>(),
    emit_set<31, 30, 21, 4>(),  emit_set<31, 31, 21, 4>(),
};

const EmitSet* find_emit(const sbf_filter* f) {
    if (f->alphabet != SBF_ALPHABET_DNA) return nullptr;
    for (const EmitSet& e : kEmitSets)
        if (e.k == static_cast<int>(f->k) && e.s == static_cast<int>(f->s) &&
            e.m == static_cast<int>(f->m) && e.h == static_cast<int>(f->h))
            return &e;
    return nullptr;
}

}  // namespace
}  // namespace sbf

extern "C" int sbf_emit_runs_async(const sbf_filter_t* f, const char* d_seq, uint64_t len,
                                   uint32_t* d_shards, uint64_t* d_masks, uint64_t capacity,
                                   uint64_t* d_count, sbf_stream_t stream) {
    using namespace sbf;
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    const EmitSet* es = find_emit(f);
    if (!es)
        return set_error(SBF_ERR_INVALID_ARGUMENT,
                         "sbf_emit_runs_async supports the DNA configurations compiled into the "
                         "library");
    if (!d_count) return set_error(SBF_ERR_INVALID_ARGUMENT, "count pointer is null");
    if (capacity && (!d_shards || !d_masks))
        return set_error(SBF_ERR_INVALID_ARGUMENT, "record buffers are null");
    if (len && !d_seq) return set_error(SBF_ERR_INVALID_ARGUMENT, "sequence pointer is null");
    if ((reinterpret_cast<uintptr_t>(d_masks) & 15u) != 0)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "mask buffer must be 16-byte aligned");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(d_count, 0, 2 * sizeof(uint64_t), st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(count)");
    const uint64_t n_kmers = f->kmers_of(len);
    if (n_kmers == 0) return SBF_OK;
    static int smem_set[64] = {};
    if (f->device >= 0 && f->device < 64 && !smem_set[f->device]) {
        for (const EmitSet& x : kEmitSets)
            if ((e = cudaFuncSetAttribute(reinterpret_cast<const void*>(x.fn),
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kEmitSmem)) != cudaSuccess)
                return cuda_fail(e, "cudaFuncSetAttribute(emit_kernel)");
        smem_set[f->device] = 1;
    }
    TileParams p{};
    p.input = reinterpret_cast<const uint8_t*>(d_seq);
    p.input_bytes = len;
    p.n_kmers = n_kmers;
    p.sym_base = 0;
    p.words = f->d_words;
    p.shard_mask = static_cast<uint32_t>(f->num_shards - 1);
    p.n_tiles = (n_kmers + kTileKmers - 1) / kTileKmers;
    p.err = f->d_err;
    RunLog log{d_shards, d_masks, capacity, reinterpret_cast<unsigned long long*>(d_count)};
    const uint64_t grid = std::min<uint64_t>(p.n_tiles, static_cast<uint64_t>(f->sms) * 2);
    es->fn<<<static_cast<unsigned>(grid), kThreads, kEmitSmem, st>>>(p, log);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "emit_kernel");
    return SBF_OK;
}

extern "C" int sbf_apply_runs_async(sbf_filter_t* f, const uint32_t* d_shards,
                                    const uint64_t* d_masks, uint64_t n, uint64_t shard_lo,
                                    uint64_t shard_hi, sbf_stream_t stream) {
    using namespace sbf;
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    if (shard_lo > shard_hi || shard_hi > f->num_shards)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "shard range [%llu, %llu) outside the filter",
                         static_cast<unsigned long long>(shard_lo),
                         static_cast<unsigned long long>(shard_hi));
    if (n == 0) return SBF_OK;
    if (!d_shards || !d_masks) return set_error(SBF_ERR_INVALID_ARGUMENT, "record buffers are null");
    if ((reinterpret_cast<uintptr_t>(d_masks) & 15u) != 0)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "mask buffer must be 16-byte aligned");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    static int ring_set[64] = {};
    cudaError_t e0;
    if (f->device >= 0 && f->device < 64 && !ring_set[f->device]) {
        if ((e0 = cudaFuncSetAttribute(reinterpret_cast<const void*>(&apply_runs_kernel),
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kInsertSlotBytes)) != cudaSuccess)
            return cuda_fail(e0, "cudaFuncSetAttribute(apply_runs_kernel)");
        ring_set[f->device] = 1;
    }
    const uint64_t blocks = std::min<uint64_t>((n + kThreads - 1) / kThreads,
                                               static_cast<uint64_t>(f->sms) * 2);
    apply_runs_kernel<<<static_cast<unsigned>(blocks), kThreads, kInsertSlotBytes, st>>>(
        d_shards, d_masks, n, f->d_words, shard_lo, shard_hi, f->d_err);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "apply_runs_kernel");
    return SBF_OK;
}

extern "C" int sbf_filter_synchronize(const sbf_filter_t* f, sbf_stream_t stream) {
    using namespace sbf;
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    return f->check_device_error(reinterpret_cast<cudaStream_t>(stream));
}
