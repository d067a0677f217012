// sbf_capi.cu -- C ABI of the Super Bloom engine (declared in include/sbf_b200.h).
//
// Host side of the drop-in boundary: it owns the filter's device words and
// staging buffers, validates arguments with the reference's rules
// (include/cusbf/filter.cuh:848-876, :1752-1782), stages host input through
// pinned double buffers so copies overlap kernels, and launches the tile
// kernels of sbf_kernels.cu.  There is no CPU fallback: every compute entry
// point runs on the GPU or fails.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/sbf_b200.h"
#include "sbf_expand.h"
#include "sbf_host.h"
#include "sbf_internal.h"

using namespace sbf;

// ---------------------------------------------------------------------------
// Error state
// ---------------------------------------------------------------------------

namespace sbf {
thread_local std::string g_last_error;
thread_local int g_last_cuda = 0;
thread_local std::string g_err_file;
thread_local uint32_t g_err_line = 0, g_err_col = 0;

void set_error_location(const char* file, uint32_t line, uint32_t col) {
    g_err_file = file ? file : "";
    g_err_line = line;
    g_err_col = col;
}

int set_error(int status, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return status;
}

int cuda_fail(cudaError_t e, const char* what) {
    g_last_cuda = static_cast<int>(e);
    return set_error(SBF_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}
}  // namespace sbf

#define SBF_CUDA(expr)                                      \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) return cuda_fail(_e, #expr); \
    } while (0)

#define SBF_TRY(expr)              \
    do {                           \
        int _s = (expr);           \
        if (_s != SBF_OK) return _s; \
    } while (0)

extern "C" const char* sbf_last_error_message(void) { return g_last_error.c_str(); }
extern "C" int sbf_last_error_location(const char** file, uint32_t* line, uint32_t* column) {
    if (file) *file = g_err_file.c_str();
    if (line) *line = g_err_line;
    if (column) *column = g_err_col;
    return SBF_OK;
}
extern "C" int sbf_last_cuda_error(void) { return g_last_cuda; }
extern "C" const char* sbf_version(void) { return "sbf-b200 0.1.0 (sm_100a)"; }

// ---------------------------------------------------------------------------
// Filter object
// ---------------------------------------------------------------------------

namespace sbf {

static uint64_t host_chunk_bytes() {
    // Host-input chunk size; a chunk is copied while the previous one is
    // hashed.  SBF_HOST_CHUNK_BYTES overrides it (minimum 4096).
    if (const char* v = std::getenv("SBF_HOST_CHUNK_BYTES")) {
        const long long b = std::strtoll(v, nullptr, 10);
        if (b > 0) return std::max<uint64_t>(static_cast<uint64_t>(b), 4096);
    }
    return uint64_t{64} << 20;
}

int Staging::ensure_device(size_t bytes) {
    if (bytes <= dev_cap) return SBF_OK;
    for (int i = 0; i < kPipeSlots; ++i) {
        if (dev[i]) cudaFree(dev[i]);
        dev[i] = nullptr;
    }
    dev_cap = 0;
    for (int i = 0; i < kPipeSlots; ++i) SBF_CUDA(cudaMalloc(&dev[i], bytes));
    dev_cap = bytes;
    return SBF_OK;
}

int Staging::ensure_pinned(size_t bytes) {
    if (bytes <= pin_cap) return SBF_OK;
    for (int i = 0; i < kPipeSlots; ++i) {
        if (pin[i]) cudaFreeHost(pin[i]);
        pin[i] = nullptr;
    }
    pin_cap = 0;
    for (int i = 0; i < kPipeSlots; ++i) SBF_CUDA(cudaMallocHost(&pin[i], bytes));
    pin_cap = bytes;
    return SBF_OK;
}

void Staging::release() {
    for (int i = 0; i < kPipeSlots; ++i) {
        if (dev[i]) cudaFree(dev[i]);
        if (pin[i]) cudaFreeHost(pin[i]);
        dev[i] = nullptr;
        pin[i] = nullptr;
    }
    dev_cap = pin_cap = 0;
}

bool is_pinned(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeManaged;
}

}  // namespace sbf

uint64_t sbf_filter::kmers_of(uint64_t symbols) const {
    return symbols < k ? 0 : symbols - k + 1;
}

int sbf_filter::require_byte_symbols(const char* what) const {
    if (width == 1) return SBF_OK;
    return set_error(SBF_ERR_INVALID_ARGUMENT,
                     "%s needs a one-byte alphabet; DNA triplets are supported by the sequence and "
                     "dense-packed entry points",
                     what);
}

int sbf_filter::launch(bool query, bool dense, const void* input, uint64_t input_bytes,
                       uint64_t n_kmers, uint8_t* out, cudaStream_t st,
                       uint32_t* out_bits) const {
    if (n_kmers == 0) return SBF_OK;
    TileParams p{};
    p.input = static_cast<const uint8_t*>(input);
    p.input_bytes = input_bytes;
    p.n_kmers = n_kmers;
    // Grid phase: aligns query output strips to 16 bytes, or the staged input
    // to 16 bytes for inserts; bit-packed queries keep phase 0 so that every
    // strip starts at a multiple of 32 windows.
    int64_t phase = 0;
    if (query && out_bits)
        phase = 0;
    else if (query)
        phase = static_cast<int64_t>(reinterpret_cast<uintptr_t>(out) & 15u);
    else if (!dense)
        phase = static_cast<int64_t>(reinterpret_cast<uintptr_t>(input) & 15u);
    p.sym_base = -phase;
    p.words = d_words;
    p.shard_mask = static_cast<uint32_t>(num_shards - 1);
    p.out = out_bits ? nullptr : out;
    p.out_bits = out_bits;
    p.n_tiles = (n_kmers + static_cast<uint64_t>(phase) + kTileKmers - 1) / kTileKmers;
    p.err = d_err;
    p.gen = gen;
    const int which = (query ? 1 : 0) + (dense ? 2 : 0);
    const void* fn = which == 0   ? ks->insert_bytes
                     : which == 1 ? ks->query_bytes
                     : which == 2 ? ks->insert_dense
                                  : ks->query_dense;
    const uint64_t resident = static_cast<uint64_t>(sms) * static_cast<uint64_t>(occupancy[which]);
    const uint64_t grid = std::min<uint64_t>(p.n_tiles, std::max<uint64_t>(resident, 1));
    SBF_CUDA(launch_set_kernel(ks, fn, static_cast<unsigned>(grid), query, p, st));
    ++launches;
    return SBF_OK;
}

int sbf_filter::check_device_error(cudaStream_t st) const {
    int h_err = 0;
    SBF_CUDA(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SBF_CUDA(cudaStreamSynchronize(st));
    if (h_err != kDevErrNone) {
        cudaMemsetAsync(d_err, 0, sizeof(int), st);
        cudaStreamSynchronize(st);
        return set_error(SBF_ERR_CUDA, "device error %d (%s)", h_err,
                         h_err == kDevErrRecordRange ? "run record outside this rank's shard range"
                                                     : "staging wait timed out");
    }
    return SBF_OK;
}

ExpandPool* sbf::host_expand_pool(sbf_filter* f) {
    if (f->expand_threads < 0) f->expand_threads = host_expand_threads();
    if (f->expand_threads == 0) return nullptr;
    if (!f->expand) {
        try {
            f->expand = new ExpandPool(f->expand_threads);
        } catch (...) {
            // No host threads to be had: download bytes from now on.
            f->expand_threads = 0;
            return nullptr;
        }
    }
    return f->expand;
}

// Host bytes -> device in chunks of whole windows with a (k-1)-symbol overlap,
// kPipeSlots chunks in flight: uploads on copy_stream, kernels on `st`,
// downloads on d2h_stream, so the three overlap across chunks.  `out_host`/`out_dev` receive query bytes.
int sbf_filter::host_pipeline(bool query, bool dense, const void* h_in, uint64_t in_bytes,
                              uint64_t n_kmers, uint8_t* out_host, uint8_t* out_dev,
                              cudaStream_t st, uint32_t* bits_host) {
    // Bit-packed results (bits_host) are written as bytes of 32-bit words:
    // chunks hold a multiple of 32 windows, so chunk c's words start at word
    // c * chunk_kmers / 32.
    const bool bits = bits_host != nullptr;
    if (n_kmers == 0) return SBF_OK;
    // Byte results for a host buffer come down one bit per window and are
    // expanded by host threads while later chunks upload (kbits: the kernel
    // writes bit-packed results).
    ExpandPool* pool = query && out_host != nullptr && !bits ? host_expand_pool(this) : nullptr;
    const bool kbits = bits || pool != nullptr;
    // Symbols <-> bytes: byte input has one byte per symbol; dense input has
    // 32 symbols per 8-byte word, so chunks are cut at word boundaries.
    const uint64_t chunk_target = host_chunk_bytes();
    uint64_t chunk_kmers;
    const uint64_t per_word = dense_per_word();
    if (dense) {
        // About chunk_target packed bytes, a whole number of words (and of
        // 32-window result words in bit-packed mode).
        const uint64_t unit = kbits ? per_word * 32 : per_word;
        const uint64_t syms = chunk_target / 8 * per_word;
        chunk_kmers = std::max<uint64_t>(syms / unit * unit, unit);
    } else {
        const uint64_t t = chunk_target / width;
        chunk_kmers = kbits ? std::max<uint64_t>(t / 32 * 32, 1024) : t;
    }
    const uint64_t n_chunks = (n_kmers + chunk_kmers - 1) / chunk_kmers;
    auto chunk_span = [&](uint64_t c, uint64_t& first_byte, uint64_t& bytes, uint64_t& kmers,
                          uint64_t& sym_offset) {
        const uint64_t w0 = c * chunk_kmers;
        kmers = std::min<uint64_t>(chunk_kmers, n_kmers - w0);
        const uint64_t syms = kmers + k - 1;
        if (dense) {
            first_byte = (w0 / per_word) * 8;
            sym_offset = w0 % per_word;  // always 0: chunk_kmers is a multiple of per_word
            bytes = std::min<uint64_t>(dense_words(sym_offset + syms) * 8, in_bytes - first_byte);
        } else {
            first_byte = w0 * width;
            sym_offset = 0;
            bytes = syms * width;
        }
    };
    const uint64_t max_in =
        dense ? dense_words(chunk_kmers + k - 1) * 8 + 8 : (chunk_kmers + k) * width;
    const bool in_pinned = is_pinned(h_in);
    if (bits) out_host = reinterpret_cast<uint8_t*>(bits_host);
    // Downloaded bytes of a chunk of `kmers` windows, and the chunk's offset
    // in the host output.
    auto out_size = [&](uint64_t kmers) { return kbits ? (kmers + 31) / 32 * 4 : kmers; };
    auto out_offset = [&](uint64_t c) { return bits ? c * chunk_kmers / 8 : c * chunk_kmers; };
    // Expanded results always pass through the pinned staging.
    const bool out_pinned = out_host != nullptr && pool == nullptr && is_pinned(out_host);
    // Moves a downloaded chunk from the pinned staging to the host output.
    auto drain = [&](uint64_t c, int slot) {
        uint64_t pf, pb, pk, po;
        chunk_span(c, pf, pb, pk, po);
        if (pool)
            pool->run(static_cast<const uint32_t*>(stage_out.pin[slot]), out_host + out_offset(c),
                      pk);
        else
            std::memcpy(out_host + out_offset(c), stage_out.pin[slot], out_size(pk));
    };
    SBF_TRY(stage_in.ensure_device(max_in));
    if (!in_pinned) SBF_TRY(stage_in.ensure_pinned(max_in));
    if (query && out_dev == nullptr) SBF_TRY(stage_out.ensure_device(out_size(chunk_kmers)));
    if (query && out_host != nullptr && !out_pinned)
        SBF_TRY(stage_out.ensure_pinned(out_size(chunk_kmers)));

    // The upload of a chunk waits for nothing but its slot; downloads run on
    // their own stream, so chunk c+1's kernel never queues behind chunk c's
    // download.
    SBF_CUDA(cudaEventRecord(ev_kernel[0], st));
    SBF_CUDA(cudaStreamWaitEvent(copy_stream, ev_kernel[0], 0));
    SBF_CUDA(cudaStreamWaitEvent(d2h_stream, ev_kernel[0], 0));
    for (uint64_t c = 0; c < n_chunks; ++c) {
        const int slot = static_cast<int>(c % kPipeSlots);
        uint64_t first_byte, bytes, kmers, sym_offset;
        chunk_span(c, first_byte, bytes, kmers, sym_offset);
        // The slot's previous kernel and download must be finished before
        // its buffers are reused.
        SBF_CUDA(cudaEventSynchronize(ev_done[slot]));
        if (query && out_host != nullptr && !out_pinned && c >= kPipeSlots)
            drain(c - kPipeSlots, slot);  // the chunk that used this slot before
        const char* src = static_cast<const char*>(h_in) + first_byte;
        if (!in_pinned) {
            std::memcpy(stage_in.pin[slot], src, bytes);
            src = static_cast<const char*>(stage_in.pin[slot]);
        }
        SBF_CUDA(cudaMemcpyAsync(stage_in.dev[slot], src, bytes, cudaMemcpyHostToDevice,
                                 copy_stream));
        SBF_CUDA(cudaEventRecord(ev_copied[slot], copy_stream));
        SBF_CUDA(cudaStreamWaitEvent(st, ev_copied[slot], 0));
        uint8_t* dout = nullptr;
        if (query) {
            dout = out_dev ? out_dev + c * chunk_kmers
                           : static_cast<uint8_t*>(stage_out.dev[slot]);
        }
        SBF_TRY(launch(query, dense, stage_in.dev[slot], bytes, kmers, kbits ? nullptr : dout, st,
                       kbits ? reinterpret_cast<uint32_t*>(dout) : nullptr));
        SBF_CUDA(cudaEventRecord(ev_kernel[slot], st));
        if (query && out_host != nullptr) {
            void* hdst = out_pinned ? static_cast<void*>(out_host + out_offset(c))
                                    : stage_out.pin[slot];
            SBF_CUDA(cudaStreamWaitEvent(d2h_stream, ev_kernel[slot], 0));
            SBF_CUDA(cudaMemcpyAsync(hdst, dout, out_size(kmers), cudaMemcpyDeviceToHost,
                                     d2h_stream));
            SBF_CUDA(cudaEventRecord(ev_done[slot], d2h_stream));
        } else {
            SBF_CUDA(cudaEventRecord(ev_done[slot], st));
        }
    }
    // `st` completes after every kernel and download of this call.
    SBF_CUDA(cudaEventRecord(ev_kernel[0], d2h_stream));
    SBF_CUDA(cudaStreamWaitEvent(st, ev_kernel[0], 0));
    if (query && out_host != nullptr && !out_pinned) {
        // The last chunks, each as soon as its download is done.
        const uint64_t first = n_chunks > kPipeSlots ? n_chunks - kPipeSlots : 0;
        for (uint64_t c = first; c < n_chunks; ++c) {
            const int slot = static_cast<int>(c % kPipeSlots);
            SBF_CUDA(cudaEventSynchronize(ev_done[slot]));
            drain(c, slot);
        }
    }
    SBF_CUDA(cudaStreamSynchronize(st));
    return check_device_error(st);
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

static inline cudaStream_t S(sbf_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

extern "C" int sbf_filter_create(uint32_t k, uint32_t s, uint32_t m, uint32_t hashes,
                                 int alphabet, uint64_t requested_bits, sbf_filter_t** out) {
    if (!out) return set_error(SBF_ERR_INVALID_ARGUMENT, "output handle pointer is null");
    *out = nullptr;
    // Symbol geometry of the alphabet (Alphabet.cuh; Config::symbolBits is
    // bit_width(symbolCount - 1), config.cuh:45-60).
    uint32_t bits = 0, width = 0;
    switch (alphabet) {
        case SBF_ALPHABET_DNA: bits = 2; width = 1; break;
        case SBF_ALPHABET_PROTEIN: bits = 5; width = 1; break;
        case SBF_ALPHABET_DNA_TRIPLET: bits = 6; width = 3; break;
        default:
            return set_error(SBF_ERR_INVALID_ARGUMENT, "unknown alphabet %d", alphabet);
    }
    // The reference's Config static_asserts (config.cuh:76-118).
    if (k == 0 || k * bits > 64)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "k=%u does not fit one packed 64-bit k-mer", k);
    if (m == 0 || m > k || s == 0 || s > k)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "need 0 < m <= k and 0 < s <= k (k=%u s=%u m=%u)",
                         k, s, m);
    if (hashes < 4 || hashes > 16 || hashes % 4 != 0)
        return set_error(SBF_ERR_INVALID_ARGUMENT,
                         "hash count %u must be 4, 8, 12 or 16 (a multiple of the 4 shard words)",
                         hashes);
    // Specialised tile kernels for the compiled DNA configurations; for any
    // other configuration, kernels compiled at run time (below, once the
    // device is known: the tile kernels for DNA, the generic kernels with
    // constant parameters for the other alphabets), or the
    // runtime-parameterised kernels when run-time compilation is not possible.
    const KernelSet* ks = alphabet == SBF_ALPHABET_DNA
                              ? find_kernels(static_cast<int>(k), static_cast<int>(s),
                                             static_cast<int>(m), static_cast<int>(hashes))
                              : nullptr;
    uint64_t blocks = requested_bits / 256 + (requested_bits % 256 != 0);
    if (blocks < 1) blocks = 1;
    uint64_t shards = 1;
    while (shards < blocks) shards <<= 1;
    auto* f = new sbf_filter();
    f->ks = ks;
    f->k = k;
    f->s = s;
    f->m = m;
    f->h = hashes;
    f->alphabet = alphabet;
    f->width = width;
    f->gen = GenericCfg{k, s, m, hashes, bits, width, static_cast<uint32_t>(alphabet)};
    f->num_shards = shards;
    f->filter_bits = shards * 256;
    int rc = SBF_OK;
    do {
        cudaError_t e = cudaGetDevice(&f->device);
        if (e != cudaSuccess) { rc = cuda_fail(e, "cudaGetDevice"); break; }
        e = cudaDeviceGetAttribute(&f->sms, cudaDevAttrMultiProcessorCount, f->device);
        if (e != cudaSuccess) { rc = cuda_fail(e, "cudaDeviceGetAttribute"); break; }
        if (!ks)
            ks = jit_kernels(static_cast<int>(k), static_cast<int>(s), static_cast<int>(m),
                             static_cast<int>(hashes), alphabet, f->device);
        if (!ks) ks = generic_kernels();
        f->ks = ks;
        const void* fns[6] = {ks->insert_bytes, ks->query_bytes, ks->insert_dense,
                              ks->query_dense, ks->insert_ragged, ks->query_ragged};
        // Run-time compiled kernels have their attributes set when loaded.
        // Their occupancy is the loaded kernel's own (registers and shared
        // memory): a persistent grid larger than what fits the SMs at once
        // runs its last CTAs as a second wave.  When the handle does not
        // answer, the set's assumption (two CTAs per SM for the tile
        // kernels, as their shared memory allows) stands.
        for (int i = 0; i < 6 && ks->jit; ++i) {
            const int dyn = ks->smem((i & 1) != 0);
            int occ = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fns[i], kThreads, dyn) !=
                    cudaSuccess ||
                occ < 1) {
                cudaGetLastError();
                occ = dyn ? std::min(ks->jit_occupancy, (227 << 10) / dyn) : ks->jit_occupancy;
            }
            f->occupancy[i] = occ;
        }
        for (int i = 0; i < 6 && rc == SBF_OK && !ks->jit; ++i) {
            // Query kernels: shard slots; insert kernels: flush staging ring.
            const int dyn = ks->smem((i & 1) != 0);
            if (dyn) {
                e = cudaFuncSetAttribute(reinterpret_cast<const void*>(fns[i]),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
                if (e != cudaSuccess) {
                    rc = cuda_fail(e, "cudaFuncSetAttribute");
                    break;
                }
            }
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&f->occupancy[i],
                                                              reinterpret_cast<const void*>(fns[i]),
                                                              kThreads, dyn);
            if (e != cudaSuccess) rc = cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
            if (f->occupancy[i] < 1) f->occupancy[i] = 1;
        }
        if (rc != SBF_OK) break;
        e = cudaMalloc(&f->d_words, shards * 32);
        if (e != cudaSuccess) {
            rc = e == cudaErrorMemoryAllocation
                     ? (cudaGetLastError(),
                        set_error(SBF_ERR_RESOURCE, "cannot allocate %llu bytes of filter words",
                                  static_cast<unsigned long long>(shards * 32)))
                     : cuda_fail(e, "cudaMalloc(words)");
            break;
        }
        e = cudaMalloc(&f->d_err, 64);
        if (e != cudaSuccess) { rc = cuda_fail(e, "cudaMalloc(err)"); break; }
        e = cudaMemset(f->d_err, 0, 64);
        if (e != cudaSuccess) { rc = cuda_fail(e, "cudaMemset(err)"); break; }
        e = cudaStreamCreateWithFlags(&f->copy_stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&f->d2h_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) { rc = cuda_fail(e, "cudaStreamCreate"); break; }
        for (int i = 0; i < kPipeSlots && rc == SBF_OK; ++i) {
            e = cudaEventCreateWithFlags(&f->ev_copied[i], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f->ev_kernel[i], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f->ev_done[i], cudaEventDisableTiming);
            if (e != cudaSuccess) rc = cuda_fail(e, "cudaEventCreate");
        }
        if (rc != SBF_OK) break;
        e = cudaMemset(f->d_words, 0, shards * 32);
        if (e != cudaSuccess) { rc = cuda_fail(e, "cudaMemset(words)"); break; }
        e = cudaDeviceSynchronize();
        if (e != cudaSuccess) { rc = cuda_fail(e, "cudaDeviceSynchronize"); break; }
    } while (false);
    if (rc != SBF_OK) {
        sbf_filter_destroy(f);
        return rc;
    }
    *out = f;
    return SBF_OK;
}

extern "C" void sbf_filter_destroy(sbf_filter_t* f) {
    if (!f) return;
    ragged_release(f);
    fastq_device_release(f);
    f->stage_in.release();
    f->stage_out.release();
    f->rb_dense.release();
    f->rb_norm.release();
    f->rb_meta.release();
    f->rb_hits.release();
    f->rb_stats.release();
    delete f->expand;
    if (f->d_words) cudaFree(f->d_words);
    if (f->d_err) cudaFree(f->d_err);
    for (int i = 0; i < kPipeSlots; ++i) {
        if (f->ev_copied[i]) cudaEventDestroy(f->ev_copied[i]);
        if (f->ev_kernel[i]) cudaEventDestroy(f->ev_kernel[i]);
        if (f->ev_done[i]) cudaEventDestroy(f->ev_done[i]);
    }
    if (f->copy_stream) cudaStreamDestroy(f->copy_stream);
    if (f->d2h_stream) cudaStreamDestroy(f->d2h_stream);
    delete f;
}

extern "C" int sbf_filter_clear(sbf_filter_t* f, sbf_stream_t stream) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    SBF_CUDA(cudaMemsetAsync(f->d_words, 0, f->num_shards * 32, S(stream)));
    SBF_CUDA(cudaStreamSynchronize(S(stream)));
    return SBF_OK;
}

extern "C" uint64_t sbf_filter_bits(const sbf_filter_t* f) { return f ? f->filter_bits : 0; }
extern "C" uint64_t sbf_filter_num_shards(const sbf_filter_t* f) { return f ? f->num_shards : 0; }

extern "C" int sbf_filter_kernel_path(const sbf_filter_t* f) {
    if (!f || !f->ks) return -1;
    return f->ks->jit ? 1 : f->ks == generic_kernels() ? 2 : 0;
}

extern "C" int sbf_filter_words(const sbf_filter_t* f, uint64_t** d_words, uint64_t* n_words) {
    if (!f || !d_words || !n_words) return set_error(SBF_ERR_INVALID_ARGUMENT, "null argument");
    *d_words = f->d_words;
    *n_words = f->num_shards * 4;
    return SBF_OK;
}

extern "C" uint64_t sbf_filter_kmer_count(const sbf_filter_t* f, uint64_t bytes) {
    return f ? f->kmers_of_bytes(bytes) : 0;
}

extern "C" int sbf_filter_load_factor(sbf_filter_t* f, sbf_stream_t stream, double* out) {
    if (!f || !out) return set_error(SBF_ERR_INVALID_ARGUMENT, "null argument");
    unsigned long long* d_count = reinterpret_cast<unsigned long long*>(f->d_err + 8);
    SBF_CUDA(launch_popcount(f->d_words, f->num_shards * 4, d_count, S(stream)));
    unsigned long long bits = 0;
    SBF_CUDA(cudaMemcpyAsync(&bits, d_count, sizeof bits, cudaMemcpyDeviceToHost, S(stream)));
    SBF_CUDA(cudaStreamSynchronize(S(stream)));
    *out = static_cast<double>(bits) / static_cast<double>(f->filter_bits);
    return SBF_OK;
}

// ---- byte sequences ---------------------------------------------------------

extern "C" int sbf_insert_sequence_async(sbf_filter_t* f, const char* d_seq, uint64_t bytes,
                                         sbf_stream_t stream, uint64_t* kmers_out) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    const uint64_t n = f->kmers_of_bytes(bytes);
    if (kmers_out) *kmers_out = n;
    if (n == 0) return SBF_OK;
    if (!d_seq) return set_error(SBF_ERR_INVALID_ARGUMENT, "sequence pointer is null");
    return f->launch(false, false, d_seq, bytes, n, nullptr, S(stream));
}

extern "C" int sbf_insert_sequence(sbf_filter_t* f, const char* h_seq, uint64_t bytes,
                                   sbf_stream_t stream, uint64_t* kmers_out) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    const uint64_t n = f->kmers_of_bytes(bytes);
    if (kmers_out) *kmers_out = n;
    if (n == 0) return SBF_OK;
    if (!h_seq) return set_error(SBF_ERR_INVALID_ARGUMENT, "sequence pointer is null");
    return f->host_pipeline(false, false, h_seq, bytes, n, nullptr, nullptr, S(stream));
}

extern "C" int sbf_contains_sequence_async(const sbf_filter_t* f, const char* d_seq,
                                           uint64_t bytes, uint8_t* d_out, uint64_t out_len,
                                           sbf_stream_t stream) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    const uint64_t n = f->kmers_of_bytes(bytes);
    if (n == 0) return SBF_OK;
    if (!d_seq || !d_out) return set_error(SBF_ERR_INVALID_ARGUMENT, "null device pointer");
    if (out_len < n)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "query output span is too small (%llu < %llu)",
                         static_cast<unsigned long long>(out_len),
                         static_cast<unsigned long long>(n));
    return f->launch(true, false, d_seq, bytes, n, d_out, S(stream));
}

extern "C" int sbf_contains_sequence_to_device(const sbf_filter_t* f, const char* h_seq,
                                               uint64_t bytes, uint8_t* d_out, uint64_t out_len,
                                               sbf_stream_t stream) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    const uint64_t n = f->kmers_of_bytes(bytes);
    if (n == 0) return SBF_OK;
    if (!h_seq || !d_out) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    if (out_len < n) return set_error(SBF_ERR_INVALID_ARGUMENT, "query output span is too small");
    return const_cast<sbf_filter*>(f)->host_pipeline(true, false, h_seq, bytes, n, nullptr, d_out,
                                                     S(stream));
}

extern "C" int sbf_contains_sequence(const sbf_filter_t* f, const char* h_seq, uint64_t bytes,
                                     uint8_t* h_out, uint64_t out_len, sbf_stream_t stream) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    const uint64_t n = f->kmers_of_bytes(bytes);
    if (n == 0) return SBF_OK;
    if (!h_seq || !h_out) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    if (out_len < n) return set_error(SBF_ERR_INVALID_ARGUMENT, "query output span is too small");
    return const_cast<sbf_filter*>(f)->host_pipeline(true, false, h_seq, bytes, n, h_out, nullptr,
                                                     S(stream));
}

// ---- bit-packed query results (no reference counterpart) ------------------------

extern "C" int sbf_contains_sequence_bits_async(const sbf_filter_t* f, const char* d_seq,
                                                uint64_t bytes, uint32_t* d_bits,
                                                uint64_t n_words, sbf_stream_t stream) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    const uint64_t n = f->kmers_of_bytes(bytes);
    if (n == 0) return SBF_OK;
    if (!d_seq || !d_bits) return set_error(SBF_ERR_INVALID_ARGUMENT, "null device pointer");
    if (reinterpret_cast<uintptr_t>(d_bits) & 3u)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "bit output must be 4-byte aligned");
    if (n_words < (n + 31) / 32)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "bit output span is too small (%llu < %llu words)",
                         static_cast<unsigned long long>(n_words),
                         static_cast<unsigned long long>((n + 31) / 32));
    return f->launch(true, false, d_seq, bytes, n, nullptr, S(stream), d_bits);
}

extern "C" int sbf_contains_sequence_bits(const sbf_filter_t* f, const char* h_seq,
                                          uint64_t bytes, uint32_t* h_bits, uint64_t n_words,
                                          sbf_stream_t stream) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    const uint64_t n = f->kmers_of_bytes(bytes);
    if (n == 0) return SBF_OK;
    if (!h_seq || !h_bits) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    if (n_words < (n + 31) / 32)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "bit output span is too small");
    return const_cast<sbf_filter*>(f)->host_pipeline(true, false, h_seq, bytes, n, nullptr,
                                                     nullptr, S(stream), h_bits);
}

// ---- dense input --------------------------------------------------------------

extern "C" int sbf_contains_dense_packed_bits_async(const sbf_filter_t* f, const uint64_t* d_words,
                                                    uint64_t n_words, uint64_t num_symbols,
                                                    uint32_t* d_bits, uint64_t n_bit_words,
                                                    sbf_stream_t stream);
extern "C" int sbf_contains_dense_packed_bits(const sbf_filter_t* f, const uint64_t* h_words,
                                              uint64_t n_words, uint64_t num_symbols,
                                              uint32_t* h_bits, uint64_t n_bit_words,
                                              sbf_stream_t stream);

extern "C" uint64_t sbf_dense_packed_word_count(uint64_t num_symbols) {
    return (num_symbols + 31) / 32;
}

extern "C" int sbf_pack_dense_device(const char* d_seq, uint64_t num_symbols, uint64_t* d_words,
                                     sbf_stream_t stream) {
    if (num_symbols == 0) return SBF_OK;
    if (!d_seq || !d_words) return set_error(SBF_ERR_INVALID_ARGUMENT, "null device pointer");
    SBF_CUDA(launch_pack_dense(reinterpret_cast<const uint8_t*>(d_seq), num_symbols, d_words,
                               S(stream)));
    return SBF_OK;
}

extern "C" int sbf_pack_dense_host(const char* h_seq, uint64_t num_symbols, uint64_t* h_words) {
    if (num_symbols == 0) return SBF_OK;
    if (!h_seq || !h_words) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    const uint64_t n_words = (num_symbols + 31) / 32;
    std::memset(h_words, 0, n_words * 8);
    for (uint64_t t = 0; t < num_symbols; ++t) {
        const uint8_t b = static_cast<uint8_t>(h_seq[t]);
        const uint8_t u = b & 0xDFu;
        const bool valid = u == 'A' || u == 'C' || u == 'G' || u == 'T';
        const uint64_t code = valid ? ((b >> 1) & 3u) : 3u;
        h_words[t / 32] |= code << (2 * (t % 32));
    }
    return SBF_OK;
}

static int check_dense(const sbf_filter_t* f, const void* words, uint64_t n_words,
                       uint64_t num_symbols) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    if (!words) return set_error(SBF_ERR_INVALID_ARGUMENT, "dense word pointer is null");
    if (n_words < f->dense_words(num_symbols))
        return set_error(SBF_ERR_INVALID_ARGUMENT, "dense packed span is too small for num_symbols");
    return SBF_OK;
}

extern "C" int sbf_insert_dense_packed_async(sbf_filter_t* f, const uint64_t* d_words,
                                             uint64_t n_words, uint64_t num_symbols,
                                             sbf_stream_t stream, uint64_t* kmers_out) {
    const uint64_t n = f ? f->kmers_of(num_symbols) : 0;
    if (kmers_out) *kmers_out = n;
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    if (n == 0) return SBF_OK;
    SBF_TRY(check_dense(f, d_words, n_words, num_symbols));
    return f->launch(false, true, d_words, f->dense_words(num_symbols) * 8, n, nullptr, S(stream));
}

extern "C" int sbf_insert_dense_packed(sbf_filter_t* f, const uint64_t* h_words,
                                       uint64_t n_words, uint64_t num_symbols, sbf_stream_t stream,
                                       uint64_t* kmers_out) {
    const uint64_t n = f ? f->kmers_of(num_symbols) : 0;
    if (kmers_out) *kmers_out = n;
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    if (n == 0) return SBF_OK;
    SBF_TRY(check_dense(f, h_words, n_words, num_symbols));
    return f->host_pipeline(false, true, h_words, f->dense_words(num_symbols) * 8, n, nullptr,
                            nullptr, S(stream));
}

extern "C" int sbf_contains_dense_packed_async(const sbf_filter_t* f, const uint64_t* d_words,
                                               uint64_t n_words, uint64_t num_symbols,
                                               uint8_t* d_out, uint64_t out_len,
                                               sbf_stream_t stream) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    const uint64_t n = f->kmers_of(num_symbols);
    if (n == 0) return SBF_OK;
    SBF_TRY(check_dense(f, d_words, n_words, num_symbols));
    if (!d_out || out_len < n)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "dense packed query output span is too small");
    return f->launch(true, true, d_words, f->dense_words(num_symbols) * 8, n, d_out, S(stream));
}

extern "C" int sbf_contains_dense_packed_to_device(const sbf_filter_t* f, const uint64_t* h_words,
                                                   uint64_t n_words, uint64_t num_symbols,
                                                   uint8_t* d_out, uint64_t out_len,
                                                   sbf_stream_t stream) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    const uint64_t n = f->kmers_of(num_symbols);
    if (n == 0) return SBF_OK;
    SBF_TRY(check_dense(f, h_words, n_words, num_symbols));
    if (!d_out || out_len < n)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "dense packed query output span is too small");
    return const_cast<sbf_filter*>(f)->host_pipeline(true, true, h_words,
                                                     f->dense_words(num_symbols) * 8, n, nullptr,
                                                     d_out, S(stream));
}

extern "C" int sbf_contains_dense_packed(const sbf_filter_t* f, const uint64_t* h_words,
                                         uint64_t n_words, uint64_t num_symbols, uint8_t* h_out,
                                         uint64_t out_len, sbf_stream_t stream) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    const uint64_t n = f->kmers_of(num_symbols);
    if (n == 0) return SBF_OK;
    SBF_TRY(check_dense(f, h_words, n_words, num_symbols));
    if (!h_out || out_len < n)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "dense packed query output span is too small");
    return const_cast<sbf_filter*>(f)->host_pipeline(true, true, h_words,
                                                     f->dense_words(num_symbols) * 8, n, h_out,
                                                     nullptr, S(stream));
}

// ---- dense input, bit-packed results (no reference counterpart) ----------------

extern "C" int sbf_contains_dense_packed_bits_async(const sbf_filter_t* f, const uint64_t* d_words,
                                                    uint64_t n_words, uint64_t num_symbols,
                                                    uint32_t* d_bits, uint64_t n_bit_words,
                                                    sbf_stream_t stream) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    const uint64_t n = f->kmers_of(num_symbols);
    if (n == 0) return SBF_OK;
    SBF_TRY(check_dense(f, d_words, n_words, num_symbols));
    if (!d_bits || (reinterpret_cast<uintptr_t>(d_bits) & 3u))
        return set_error(SBF_ERR_INVALID_ARGUMENT, "bit output must be a 4-byte aligned pointer");
    if (n_bit_words < (n + 31) / 32)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "bit output span is too small");
    return f->launch(true, true, d_words, f->dense_words(num_symbols) * 8, n, nullptr, S(stream),
                     d_bits);
}

extern "C" int sbf_contains_dense_packed_bits(const sbf_filter_t* f, const uint64_t* h_words,
                                              uint64_t n_words, uint64_t num_symbols,
                                              uint32_t* h_bits, uint64_t n_bit_words,
                                              sbf_stream_t stream) {
    if (!f) return set_error(SBF_ERR_INVALID_ARGUMENT, "filter is null");
    const uint64_t n = f->kmers_of(num_symbols);
    if (n == 0) return SBF_OK;
    SBF_TRY(check_dense(f, h_words, n_words, num_symbols));
    if (!h_bits || n_bit_words < (n + 31) / 32)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "bit output span is too small");
    return const_cast<sbf_filter*>(f)->host_pipeline(true, true, h_words,
                                                     f->dense_words(num_symbols) * 8, n, nullptr,
                                                     nullptr, S(stream), h_bits);
}
