// sbf_kernels.cu -- the tile kernels compiled for the common configurations
// (the kernel is in sbf_tile.cuh; other DNA configurations are compiled at
// run time by sbf_jit.cpp) and the auxiliary kernels.
#include <cuda_runtime.h>

#include <cstdint>

#include "sbf_device.cuh"
#include "sbf_internal.h"
#include "sbf_tile.cuh"

namespace sbf {

// tile_rec[t] = first record whose end exceeds the first byte tile t stages
// (binary search; records sorted and non-overlapping).
__global__ void tile_records_kernel(const DevRange* ranges, uint64_t n, int64_t sym_base,
                                    uint64_t n_tiles, uint32_t* tile_rec) {
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n_tiles) return;
    const int64_t s0 = static_cast<int64_t>(t) * kTileKmers + sym_base;
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (static_cast<int64_t>(ranges[mid].offset + ranges[mid].bytes) > s0)
            hi = mid;
        else
            lo = mid + 1;
    }
    tile_rec[t] = static_cast<uint32_t>(lo);
}

// tile_records_kernel with the record and tile counts read on the device.
__global__ void tile_records_sized_kernel(const DevRange* ranges, const DevSizes* sizes,
                                          int64_t sym_base, uint32_t* tile_rec) {
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= sizes->n_tiles) return;
    const uint64_t n = sizes->n_ranges;
    const int64_t s0 = static_cast<int64_t>(t) * kTileKmers + sym_base;
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (static_cast<int64_t>(ranges[mid].offset + ranges[mid].bytes) > s0)
            hi = mid;
        else
            lo = mid + 1;
    }
    tile_rec[t] = static_cast<uint32_t>(lo);
}

// ---------------------------------------------------------------------------
// Auxiliary kernels
// ---------------------------------------------------------------------------

// Dense packing: 32 symbols per word, symbol t at bits [2t, 2t+2), invalid
// bytes stored as their low two code bits (include/cusbf/dense_packed.hpp:26-50).
__global__ void pack_dense_kernel(const uint8_t* seq, uint64_t num_symbols, uint64_t* words) {
    const uint64_t w = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t n_words = (num_symbols + 31) / 32;
    if (w >= n_words) return;
    const uint64_t first = w * 32;
    uint64_t out = 0;
    for (int t = 0; t < 32; ++t) {
        const uint64_t s = first + t;
        if (s >= num_symbols) break;
        const uint8_t b = seq[s];
        const uint8_t upper = b & 0xDFu;
        const bool valid = upper == 'A' || upper == 'C' || upper == 'G' || upper == 'T';
        const uint64_t code = valid ? ((b >> 1) & 3u) : 3u;
        out |= code << (2 * t);
    }
    words[w] = out;
}

__global__ void popcount_kernel(const uint64_t* words, uint64_t n, unsigned long long* out) {
    unsigned long long local = 0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        local += __popcll(words[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xFFFFFFFFu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(out, local);
}

cudaError_t launch_pack_dense(const uint8_t* seq, uint64_t num_symbols, uint64_t* words,
                              cudaStream_t stream) {
    const uint64_t n_words = (num_symbols + 31) / 32;
    if (n_words == 0) return cudaSuccess;
    pack_dense_kernel<<<static_cast<unsigned>((n_words + 255) / 256), 256, 0, stream>>>(
        seq, num_symbols, words);
    return cudaGetLastError();
}

const void* tile_records_kernel_ptr() { return reinterpret_cast<const void*>(&tile_records_kernel); }

cudaError_t launch_tile_records(const DevRange* ranges, uint64_t n_ranges, int64_t sym_base,
                                uint64_t n_tiles, uint32_t* tile_rec, cudaStream_t stream) {
    if (n_tiles == 0) return cudaSuccess;
    tile_records_kernel<<<static_cast<unsigned>((n_tiles + 255) / 256), 256, 0, stream>>>(
        ranges, n_ranges, sym_base, n_tiles, tile_rec);
    return cudaGetLastError();
}

cudaError_t launch_tile_records_sized(const DevRange* ranges, const DevSizes* sizes,
                                      int64_t sym_base, uint64_t max_tiles, uint32_t* tile_rec,
                                      cudaStream_t stream) {
    if (max_tiles == 0) return cudaSuccess;
    tile_records_sized_kernel<<<static_cast<unsigned>((max_tiles + 255) / 256), 256, 0, stream>>>(
        ranges, sizes, sym_base, tile_rec);
    return cudaGetLastError();
}

cudaError_t launch_popcount(const uint64_t* words, uint64_t n_words, unsigned long long* out,
                            cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    if (n_words == 0) return cudaSuccess;
    uint64_t blocks = (n_words + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    popcount_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(words, n_words, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Compiled configurations
// ---------------------------------------------------------------------------

template <class Fn>
const void* fn_ptr(Fn* f) {
    return reinterpret_cast<const void*>(f);
}

template <int K, int S, int M, int H>
KernelSet make_set() {
    using C = Cfg<K, S, M, H>;
    return KernelSet{K,
                     S,
                     M,
                     H,
                     fn_ptr(&tile_kernel<C, false, false, false>),
                     fn_ptr(&tile_kernel<C, true, false, false>),
                     fn_ptr(&tile_kernel<C, false, true, false>),
                     fn_ptr(&tile_kernel<C, true, true, false>),
                     fn_ptr(&tile_kernel<C, false, false, true>),
                     fn_ptr(&tile_kernel<C, true, false, true>)};
}

static const KernelSet kSets[] = {
    make_set<31, 28, 16, 4>(),  // the benchmark configuration
    make_set<31, 30, 16, 4>(),  make_set<31, 31, 16, 4>(), make_set<31, 28, 16, 8>(),
    make_set<31, 28, 16, 16>(), make_set<21, 19, 11, 4>(), make_set<5, 4, 3, 4>(),
    make_set<3, 2, 2, 4>(),
    // The reference's FPR sweep over s (benchmarks/fpr_fastx_sweep.cu:294-302).
    make_set<31, 28, 21, 4>(), make_set<31, 30, 21, 4>(), make_set<31, 31, 21, 4>(),
};

const KernelSet* find_kernels(int k, int s, int m, int h) {
    for (const KernelSet& ks : kSets)
        if (ks.k == k && ks.s == s && ks.m == m && ks.h == h) return &ks;
    return nullptr;
}

cudaError_t launch_set_kernel(const KernelSet* ks, const void* fn, unsigned grid, bool query,
                              const TileParams& p, cudaStream_t stream) {
    TileParams copy = p;
    void* args[] = {&copy};
    return cudaLaunchKernel(fn, dim3(grid), dim3(kThreads), args, ks->smem(query), stream);
}

}  // namespace sbf
