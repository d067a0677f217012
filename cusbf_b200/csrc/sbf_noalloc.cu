// sbf_noalloc.cu -- per-record counts of a device record batch without any
// allocation: sbf_record_batch_counts_noalloc.
//
// For callers that may not allocate device memory at call time: a serving
// loop whose device memory is reserved once at start-up and must not grow
// while requests are in flight, or an allocator hook that must not re-enter
// the CUDA allocator it is part of.  The other record batch entry points keep
// grow-only device buffers inside the filter and may cudaMalloc when a batch
// is larger than any before it; this one uses only a fixed 8 MiB scratch area
// compiled into the library.  It is synchronous: it copies the caller's host
// range table in and the counts out, and returns once its stream has reached
// the end of the call.
//
// The counts are those of the reference's valid_record_kmer_count
// (include/cusbf/normalized_record_batch.hpp:88-110) and
// count_positive_kmers_per_record (include/cusbf/detail/count_positive_kmers.cuh:21-45),
// i.e. the queried_kmers / positive_kmers of each record of query_record_batch.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/sbf_b200.h"
#include "sbf_host.h"
#include "sbf_internal.h"

namespace sbf {


namespace {

// Scratch: [ranges: n x 16 B][valid: n x 8 B][positive: n x 8 B].
constexpr uint64_t kNoAllocScratchBytes = 8ull << 20;
constexpr uint64_t kNoAllocBytesPerRecord =
    sizeof(sbf_record_range) + 2 * sizeof(unsigned long long);
constexpr uint64_t kNoAllocMaxRecords = kNoAllocScratchBytes / kNoAllocBytesPerRecord;
static_assert(kNoAllocMaxRecords == 262144, "scratch layout changed");

__device__ __align__(256) unsigned char g_count_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

__device__ __forceinline__ bool dna_byte_valid(uint8_t b) {
    const uint8_t u = b & 0xDFu;
    return u == 'A' || u == 'C' || u == 'G' || u == 'T';
}

// One warp per record (grid-strided).  Window p of a record is valid iff its
// K bytes are all A/C/G/T; positives are the set hit bytes of its windows.
// Every record's two counters are written with plain stores by the one warp
// that owns the record, so nothing in the scratch has to start at zero.
__global__ void record_counts_kernel(const uint8_t* seq, const sbf_record_range* ranges,
                                     uint64_t n, uint32_t k, const uint8_t* hits,
                                     unsigned long long* valid_out,
                                     unsigned long long* positive_out) {
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t warps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t r = warp; r < n; r += warps) {
        const uint64_t off = ranges[r].sequence_offset;
        const uint64_t size = ranges[r].sequence_bytes;
        unsigned long long valid = 0, pos = 0;
        if (size >= k) {
            const uint8_t* rec = seq + off;
            const uint64_t windows = size - k + 1;
            // Scan window ends e in [k-1, size), tracking the last invalid byte.
            int64_t last_inv = -1;
            for (uint64_t base = 0; base < size; base += 32) {
                const uint64_t e = base + lane;
                const bool in = e < size;
                const bool inv = in && !dna_byte_valid(rec[e]);
                const uint32_t m = __ballot_sync(0xFFFFFFFFu, inv);
                const uint32_t upto = m & (0xFFFFFFFFu >> (31 - lane));
                const int64_t li =
                    upto ? static_cast<int64_t>(base) + (31 - __clz(upto)) : last_inv;
                const bool ok = in && e + 1 >= k && static_cast<int64_t>(e) - li >= k;
                valid += __popc(__ballot_sync(0xFFFFFFFFu, ok));
                if (m) last_inv = static_cast<int64_t>(base) + (31 - __clz(m));
            }
            if (hits) {
                const uint8_t* h = hits + off;
                unsigned long long local = 0;
                for (uint64_t p = lane; p < windows; p += 32) local += h[p];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xFFFFFFFFu, local, o);
                pos = local;
            }
        }
        if (lane == 0) {
            valid_out[r] = valid;
            positive_out[r] = pos;
        }
    }
}

// Device address of the scratch on `device`, looked up once per device with
// that device current (the first call on a device does the lookup).
int scratch_for(int device, void** out) {
    if (device < 0 || device >= kMaxDevices)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "device ordinal %d out of range", device);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[device]) {
        int current = 0;
        cudaError_t e = cudaGetDevice(&current);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
        if (current != device && (e = cudaSetDevice(device)) != cudaSuccess)
            return cuda_fail(e, "cudaSetDevice");
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_count_scratch);
        if (current != device) {
            const cudaError_t r = cudaSetDevice(current);
            if (r != cudaSuccess) return cuda_fail(r, "cudaSetDevice (restoring the caller's device)");
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_count_scratch)");
        g_scratch_ptr[device] = p;
    }
    *out = g_scratch_ptr[device];
    return SBF_OK;
}

}  // namespace
}  // namespace sbf

extern "C" int sbf_record_batch_counts_noalloc(const sbf_filter_t* f, const char* d_seq,
                                               uint64_t len, const sbf_record_range* ranges,
                                               uint64_t n, const uint8_t* d_hits,
                                               uint64_t hits_len, sbf_stream_t stream,
                                               uint64_t* valid_out, uint64_t* positive_out) {
    using namespace sbf;
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    if (f->alphabet != SBF_ALPHABET_DNA)
        return set_error(SBF_ERR_INVALID_ARGUMENT,
                         "sbf_record_batch_counts_noalloc counts DNA windows only");
    if (n && (!ranges || !valid_out || !positive_out))
        return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    if (n > kNoAllocMaxRecords)
        return set_error(SBF_ERR_INVALID_ARGUMENT,
                         "record batch of %llu records exceeds the %llu-record limit of "
                         "sbf_record_batch_counts_noalloc (%llu bytes of static scratch)",
                         static_cast<unsigned long long>(n),
                         static_cast<unsigned long long>(kNoAllocMaxRecords),
                         static_cast<unsigned long long>(kNoAllocScratchBytes));
    int s = validate_ranges(len, ranges, n);
    if (s != SBF_OK) return s;
    if (n == 0) return SBF_OK;
    if (!d_seq && len) return set_error(SBF_ERR_INVALID_ARGUMENT, "sequence pointer is null");
    const uint64_t windows = f->kmers_of(len);
    if (d_hits && hits_len < windows)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "hit span is shorter than the batch's windows");
    // The scratch address and the launch below belong to the filter's device,
    // so that device must be the caller's current one.
    int current = -1;
    cudaError_t e = cudaGetDevice(&current);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (current != f->device)
        return set_error(SBF_ERR_INVALID_ARGUMENT,
                         "sbf_record_batch_counts_noalloc: the current device (%d) is not the "
                         "filter's device (%d)",
                         current, f->device);
    void* scratch = nullptr;
    if ((s = scratch_for(f->device, &scratch)) != SBF_OK) return s;
    auto* d_ranges = static_cast<sbf_record_range*>(scratch);
    auto* d_valid = reinterpret_cast<unsigned long long*>(d_ranges + n);
    auto* d_pos = d_valid + n;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    e = cudaMemcpyAsync(d_ranges, ranges, n * sizeof(sbf_record_range), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(ranges)");
    const uint64_t warps = n < static_cast<uint64_t>(f->sms) * 64 ? n : static_cast<uint64_t>(f->sms) * 64;
    record_counts_kernel<<<static_cast<unsigned>((warps * 32 + 255) / 256), 256, 0, st>>>(
        reinterpret_cast<const uint8_t*>(d_seq), d_ranges, n, f->k, d_hits, d_valid, d_pos);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "record_counts_kernel");
    if ((e = cudaMemcpyAsync(valid_out, d_valid, n * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyAsync(valid)");
    if ((e = cudaMemcpyAsync(positive_out, d_pos, n * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyAsync(positive)");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    return SBF_OK;
}
