// sbf_persist.cu -- filter persistence: the shard words with a small header,
// written to and read from a file.  No reference counterpart (the reference
// keeps filters in device memory only); the word layout is the reference's
// filter_block array (include/cusbf/detail/filter_impl.cuh:19-48), so a saved
// file is also the artefact that parity checks compare.
//
// File layout (little-endian):
//   bytes  0..7   magic "SBFB200\0"
//   bytes  8..11  format version (1)
//   bytes 12..27  k, s, m, hashes (uint32 each)
//   bytes 28..31  alphabet id
//   bytes 32..39  num_shards (uint64)
//   bytes 40..    num_shards * 32 bytes of shard words
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <sys/types.h>

#include "../../include/sbf_b200.h"
#include "sbf_host.h"

using namespace sbf;

namespace {

constexpr char kMagic[8] = {'S', 'B', 'F', 'B', '2', '0', '0', '\0'};
constexpr uint32_t kVersion = 1;
constexpr uint64_t kChunk = uint64_t{64} << 20;

struct Header {
    char magic[8];
    uint32_t version;
    uint32_t k, s, m, h;
    uint32_t alphabet;
    uint64_t num_shards;
};
static_assert(sizeof(Header) == 40, "header layout");

struct File {
    std::FILE* fp = nullptr;
    ~File() {
        if (fp) std::fclose(fp);
    }
};

struct Pinned {
    void* p = nullptr;
    ~Pinned() {
        if (p) cudaFreeHost(p);
    }
};

int io_error(const char* what, const char* path) {
    return set_error(SBF_ERR_IO, "%s '%s' failed", what, path);
}

}  // namespace

extern "C" int sbf_filter_save(const sbf_filter_t* f, const char* path, sbf_stream_t stream) {
    if (!f || !path) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    File file;
    file.fp = std::fopen(path, "wb");
    if (!file.fp) return io_error("opening", path);
    Header hd{};
    std::memcpy(hd.magic, kMagic, sizeof kMagic);
    hd.version = kVersion;
    hd.k = f->k;
    hd.s = f->s;
    hd.m = f->m;
    hd.h = f->h;
    hd.alphabet = SBF_ALPHABET_DNA;
    hd.num_shards = f->num_shards;
    if (std::fwrite(&hd, sizeof hd, 1, file.fp) != 1) return io_error("writing", path);
    const uint64_t total = f->num_shards * 32;
    Pinned buf;
    cudaError_t e = cudaMallocHost(&buf.p, std::min(total, kChunk));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const auto* src = reinterpret_cast<const uint8_t*>(f->d_words);
    for (uint64_t off = 0; off < total; off += kChunk) {
        const uint64_t n = std::min(kChunk, total - off);
        if ((e = cudaMemcpyAsync(buf.p, src + off, n, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return cuda_fail(e, "cudaMemcpyAsync(words)");
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
        if (std::fwrite(buf.p, 1, n, file.fp) != n) return io_error("writing", path);
    }
    if (std::fflush(file.fp) != 0) return io_error("flushing", path);
    return SBF_OK;
}

extern "C" int sbf_filter_file_info(const char* path, uint32_t* k, uint32_t* s, uint32_t* m,
                                    uint32_t* hashes, uint64_t* filter_bits) {
    if (!path) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    File file;
    file.fp = std::fopen(path, "rb");
    if (!file.fp) return io_error("opening", path);
    Header hd{};
    if (std::fread(&hd, sizeof hd, 1, file.fp) != 1 || std::memcmp(hd.magic, kMagic, 8) != 0)
        return set_error(SBF_ERR_IO, "'%s' is not a saved filter", path);
    if (hd.version != kVersion)
        return set_error(SBF_ERR_IO, "'%s' has format version %u (expected %u)", path,
                         hd.version, kVersion);
    if (k) *k = hd.k;
    if (s) *s = hd.s;
    if (m) *m = hd.m;
    if (hashes) *hashes = hd.h;
    if (filter_bits) *filter_bits = hd.num_shards * 256;
    return SBF_OK;
}

extern "C" int sbf_filter_load(sbf_filter_t* f, const char* path, sbf_stream_t stream) {
    if (!f || !path) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    File file;
    file.fp = std::fopen(path, "rb");
    if (!file.fp) return io_error("opening", path);
    Header hd{};
    if (std::fread(&hd, sizeof hd, 1, file.fp) != 1 || std::memcmp(hd.magic, kMagic, 8) != 0)
        return set_error(SBF_ERR_IO, "'%s' is not a saved filter", path);
    if (hd.version != kVersion)
        return set_error(SBF_ERR_IO, "'%s' has format version %u (expected %u)", path,
                         hd.version, kVersion);
    if (hd.k != f->k || hd.s != f->s || hd.m != f->m || hd.h != f->h ||
        hd.alphabet != SBF_ALPHABET_DNA || hd.num_shards != f->num_shards)
        return set_error(SBF_ERR_INVALID_ARGUMENT,
                         "'%s' holds a filter of k=%u s=%u m=%u hashes=%u with %llu shards; "
                         "this filter has k=%u s=%u m=%u hashes=%u with %llu shards",
                         path, hd.k, hd.s, hd.m, hd.h,
                         static_cast<unsigned long long>(hd.num_shards), f->k, f->s, f->m, f->h,
                         static_cast<unsigned long long>(f->num_shards));
    const uint64_t total = f->num_shards * 32;
    // Check the size first, so a short or long file leaves the filter as it was.
    if (fseeko(file.fp, 0, SEEK_END) != 0) return io_error("seeking", path);
    const off_t size = ftello(file.fp);
    if (size < 0 || static_cast<uint64_t>(size) != sizeof(Header) + total)
        return set_error(SBF_ERR_IO, "'%s' has %lld bytes; a filter of %llu shards needs %llu",
                         path, static_cast<long long>(size),
                         static_cast<unsigned long long>(f->num_shards),
                         static_cast<unsigned long long>(sizeof(Header) + total));
    if (fseeko(file.fp, sizeof(Header), SEEK_SET) != 0) return io_error("seeking", path);
    Pinned buf;
    cudaError_t e = cudaMallocHost(&buf.p, std::min(total, kChunk));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    auto* dst = reinterpret_cast<uint8_t*>(f->d_words);
    for (uint64_t off = 0; off < total; off += kChunk) {
        const uint64_t n = std::min(kChunk, total - off);
        if (std::fread(buf.p, 1, n, file.fp) != n)
            return set_error(SBF_ERR_IO, "'%s' is truncated", path);
        if ((e = cudaMemcpyAsync(dst + off, buf.p, n, cudaMemcpyHostToDevice, st)) != cudaSuccess)
            return cuda_fail(e, "cudaMemcpyAsync(words)");
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    }
    return SBF_OK;
}
