// test_cpp_api.cu -- the C++ drop-in headers (include/cusbf/*) compiled as a
// caller of the reference API would use them, with checks restating the
// reference's GPU unit tests (tests/test_bloom_filter.cu, tests/test_fastx.cu
// of tdortman/cuSBF, Config<5,4,3,4>).  Built by tests/test_cpp_api.py; exits
// non-zero on the first failed check.
#include <array>
#include <cstdio>
#include <cstdlib>
#include <sstream>
#include <string>
#include <vector>

#include <cusbf/dense_packed.hpp>
#include <cusbf/detail/query_layout.cuh>
#include <cusbf/filter.cuh>

using TestConfig = cusbf::Config<5, 4, 3, 4>;
using K31 = cusbf::Config<31, 28, 16, 4>;

static int failures = 0;
#define CHECK(cond)                                                      \
    do {                                                                 \
        if (!(cond)) {                                                   \
            std::fprintf(stderr, "%s:%d: CHECK(%s)\n", __FILE__, __LINE__, #cond); \
            ++failures;                                                  \
        }                                                                \
    } while (0)

// A caller's own kernels over filter::ref(), as the reference's device view
// allows (filter_ref.cuh:70-108): window i of a DNA sequence is packed
// MSB-first (A0 C1 T2 G3), its minimizer selects the shard, and the window is
// tested with sectorized_contains_packed_kmer or inserted with
// apply_word_masks.
__device__ uint32_t user_dna_code(char c) {
    switch (c & 0xDF) {
        case 'A': return 0;
        case 'C': return 1;
        case 'T': return 2;
        case 'G': return 3;
        default: return 0xFFu;
    }
}

template <class Cfg>
__device__ bool user_window(const char* seq, uint64_t i, uint64_t& packed, uint64_t& minhash) {
    bool valid = true;
    packed = 0;
    for (int j = 0; j < Cfg::k; ++j) {
        const uint32_t c = user_dna_code(seq[i + j]);
        valid &= c != 0xFFu;
        packed = (packed << 2) | (c & 3u);
    }
    minhash = ~uint64_t{0};
    for (int o = 0; o + Cfg::m <= Cfg::k; ++o) {
        const uint64_t mm = (packed >> (2 * (Cfg::k - o - Cfg::m))) & ((uint64_t{1} << (2 * Cfg::m)) - 1);
        const uint64_t h = mm * 0x9E3779B97F4A7C15ULL;
        minhash = h < minhash ? h : minhash;
    }
    return valid;
}

template <class Cfg>
__global__ void user_query(cusbf::filter_ref<Cfg> ref, const char* seq, uint64_t n, uint8_t* out) {
    const uint64_t i = blockIdx.x * uint64_t{blockDim.x} + threadIdx.x;
    if (i >= n) return;
    uint64_t packed, minhash;
    const bool valid = user_window<Cfg>(seq, i, packed, minhash);
    const auto& block = ref.blocks()[ref.shard_index(minhash)];
    out[i] = valid && cusbf::filter_ref<Cfg>::sectorized_contains_packed_kmer(packed, block.words);
}

template <class Cfg>
__global__ void user_insert(cusbf::filter_ref<Cfg> ref, const char* seq, uint64_t n) {
    const uint64_t i = blockIdx.x * uint64_t{blockDim.x} + threadIdx.x;
    if (i >= n) return;
    uint64_t packed, minhash;
    if (!user_window<Cfg>(seq, i, packed, minhash)) return;
    uint64_t m[4] = {0, 0, 0, 0};
    for (int o = 0; o + Cfg::s <= Cfg::k; ++o) {
        uint64_t h = ((packed >> (2 * (Cfg::k - o - Cfg::s))) & ((uint64_t{1} << (2 * Cfg::s)) - 1)) *
                     0x9e3779b97f4a7c15ULL;
        h ^= h >> 33;
        for (uint64_t j = 0; j < Cfg::hashCount; ++j)
            m[j % 4] |= uint64_t{1} << cusbf::filter_block<Cfg>::sectorizedBitAddress(h, j);
    }
    ref.apply_word_masks(ref.blocks()[ref.shard_index(minhash)], m[0], m[1], m[2], m[3]);
}

static bool all_ones(const std::vector<uint8_t>& v) {
    for (uint8_t x : v)
        if (x != 1) return false;
    return true;
}

int main() {
    {  // test_bloom_filter.cu:10-20
        cusbf::filter<TestConfig> f(1 << 12);
        const std::string seq = "ACGTACGTACGTACGT";
        const uint64_t n = CUSBF_UNWRAP(f.insert_sequence(seq));
        const auto hits = CUSBF_UNWRAP(f.contains_sequence(seq));
        CHECK(n == seq.size() - TestConfig::k + 1);
        CHECK(hits.size() == n && all_ones(hits));
        const float lf = f.load_factor();
        (void)CUSBF_UNWRAP(f.insert_sequence(seq));
        CHECK(lf == f.load_factor());
        (void)CUSBF_UNWRAP(f.clear());
        const auto after = CUSBF_UNWRAP(f.contains_sequence(seq));
        for (uint8_t x : after) CHECK(x == 0);
    }
    {  // :91-101
        cusbf::filter<TestConfig> f(1 << 12);
        const std::string seq = "ACGTNACGTACGTA";
        (void)CUSBF_UNWRAP(f.insert_sequence(seq));
        const auto hits = CUSBF_UNWRAP(f.contains_sequence(seq));
        CHECK((hits == std::vector<uint8_t>{0, 0, 0, 0, 0, 1, 1, 1, 1, 1}));
    }
    {  // :22-38 dense == byte path
        cusbf::filter<TestConfig> f(1 << 12);
        const std::string seq = "ACGTACGTACGTACGTACGTACGT";
        const auto packed = cusbf::pack_dense_sequence<TestConfig>(seq);
        CHECK(CUSBF_UNWRAP(f.insert_dense_packed(packed, seq.size())) == seq.size() - 4);
        const auto dh = CUSBF_UNWRAP(f.contains_dense_packed(packed, seq.size()));
        CHECK(all_ones(dh) && dh == CUSBF_UNWRAP(f.contains_sequence(seq)));
    }
    {  // :342-422 device record batch and separator windows
        cusbf::filter<TestConfig> f(1 << 14);
        const std::string r1 = "ACGTACGTACGT", r2 = "TTGGAACCTTGG";
        const std::string joined = r1 + "N" + r2;
        char* d = nullptr;
        uint8_t* out = nullptr;
        CUSBF_CUDA_CALL(cudaMalloc(&d, joined.size()));
        CUSBF_CUDA_CALL(cudaMalloc(&out, 21));
        CUSBF_CUDA_CALL(cudaMemcpy(d, joined.data(), joined.size(), cudaMemcpyHostToDevice));
        const std::array<cusbf::RecordRange, 2> ranges{{{0, 12}, {13, 12}}};
        CHECK(CUSBF_UNWRAP(f.insert_record_batch_async(
                  cusbf::device_span<const char>{d, joined.size()}, ranges)) == 16);
        CUSBF_CUDA_CALL(cudaDeviceSynchronize());
        cusbf::filter<TestConfig> g(1 << 14);
        (void)CUSBF_UNWRAP(g.insert_sequence(r1));
        (void)CUSBF_UNWRAP(g.insert_sequence(r2));
        cusbf::require_void(g.contains_record_batch_async(
            cusbf::device_span<const char>{d, joined.size()}, ranges,
            cusbf::device_span<uint8_t>{out, 21}));
        std::vector<uint8_t> hits(21);
        CUSBF_CUDA_CALL(cudaMemcpy(hits.data(), out, 21, cudaMemcpyDeviceToHost));
        std::vector<uint8_t> want(21, 1);
        for (int i = 8; i < 13; ++i) want[i] = 0;
        CHECK(hits == want);
        const auto bad = g.contains_record_batch_async(
            cusbf::device_span<const char>{d, joined.size()}, ranges,
            cusbf::device_span<uint8_t>{out, 20});
        CHECK(!bad && bad.error().category() == cusbf::ErrorCategory::invalid_argument);
        cudaFree(d);
        cudaFree(out);
    }
    {  // test_fastx.cu:576-666 forced chunk flush
        cusbf::filter<TestConfig> f(1 << 12);
        const std::string text = ">first\nACGTACGT\n>second\nACGTNACGTACGTA\n>third\nTGCATGCA\n";
        std::istringstream ins(text);
        const auto rep = CUSBF_UNWRAP(f.insert_fastx(ins, 0.0));
        CHECK(rep.recordsIndexed == 3 && rep.indexedBases == 30 && rep.insertedKmers == 13);
        std::istringstream qs(text);
        const auto det = CUSBF_UNWRAP(f.query_fastx_detailed(qs, 0.0));
        CHECK(det.records.size() == 3 && det.summary.positive_kmers == 13);
        CHECK(det.records[1].header == "second");
        CHECK((det.records[1].hits == std::vector<uint8_t>{0, 0, 0, 0, 0, 1, 1, 1, 1, 1}));
        // A throwing consumer stops the query and the filter stays usable
        // (test_fastx.cu:728-826).
        std::istringstream qa(text);
        int calls = 0;
        bool thrown = false;
        try {
            (void)f.query_fastx_records(qa, [&](const cusbf::FastxRecordView&) {
                if (++calls == 2) throw std::runtime_error("stop");
            });
        } catch (const std::runtime_error&) {
            thrown = true;
        }
        CHECK(thrown && calls == 2);
        std::istringstream qb(text);
        CHECK(CUSBF_UNWRAP(f.query_fastx(qb)).positive_kmers == 13);
        std::istringstream broken("@broken\nACGTACGT\n+\nIIIIIII\n");
        const auto err = f.query_fastx(broken);
        CHECK(!err && err.error().category() == cusbf::ErrorCategory::fastx_parse);
        CHECK(err.error().as_fastx_parse()->location.line == 4);
        CHECK(err.error().as_fastx_parse()->location.column == 8);
    }
    {  // test_query_layout.cpp / test_normalized_record_batch.cpp (host)
        using C3 = cusbf::Config<3, 2, 2, 4>;
        const std::array<cusbf::NormalizedRecord, 2> recs{{{0, 0, 6, 1}, {1, 6, 8, 2}}};
        const auto layout = cusbf::detail::QueryLayout::build<C3>(recs);
        CHECK(layout.total_hit_count() == 13 && layout.records()[1].hit_offset == 7);
        const std::array<cusbf::RecordRange, 2> ranges{{{0, 4}, {4, 4}}};
        const auto nb = CUSBF_UNWRAP(
            cusbf::normalize_record_batch<C3>(cusbf::RecordBatchView{"ACGTACGTACGT", ranges}));
        CHECK(nb.sequence() == "ACGTNACGT" && nb.total_valid_kmers() == 4);
        const std::array<cusbf::RecordRange, 2> overlap{{{4, 4}, {0, 4}}};
        const auto e = cusbf::normalize_record_batch<C3>(cusbf::RecordBatchView{"ACGTACGT", overlap});
        CHECK(!e && e.error().category() == cusbf::ErrorCategory::invalid_argument);
    }
    {  // k = 31 engine words through the C++ interface
        cusbf::filter<K31> f(1 << 20);
        std::string seq(5000, 'A');
        uint64_t x = 88172645463325252ull;
        for (char& c : seq) {
            x ^= x << 13;
            x ^= x >> 7;
            x ^= x << 17;
            c = "ACGT"[x & 3];
        }
        CHECK(CUSBF_UNWRAP(f.insert_sequence(seq)) == 5000 - 30);
        CHECK(all_ones(CUSBF_UNWRAP(f.contains_sequence(seq))));
        CHECK(f.num_shards() == (1u << 12) && f.filter_bits() == (1u << 20));
        CHECK(f.ref().num_blocks() == f.num_shards());
    }
    {  // filter_ref device members from a caller's kernels (filter_ref.cuh:70-108)
        cusbf::filter<K31> f(1 << 22), g(1 << 22);
        std::string seq(40000, 'A');
        uint64_t x = 0x9E3779B97F4A7C15ull;
        for (size_t i = 0; i < seq.size(); ++i) {
            x ^= x << 13;
            x ^= x >> 7;
            x ^= x << 17;
            seq[i] = (i % 997 == 5) ? 'N' : "ACGTacgt"[x & 7];
        }
        const uint64_t n = seq.size() - K31::k + 1;
        (void)CUSBF_UNWRAP(f.insert_sequence(seq.substr(0, 25000)));
        const auto want = CUSBF_UNWRAP(f.contains_sequence(seq));
        char* d = nullptr;
        uint8_t* out = nullptr;
        CUSBF_CUDA_CALL(cudaMalloc(&d, seq.size()));
        CUSBF_CUDA_CALL(cudaMalloc(&out, n));
        CUSBF_CUDA_CALL(cudaMemcpy(d, seq.data(), seq.size(), cudaMemcpyHostToDevice));
        user_query<K31><<<(n + 255) / 256, 256>>>(f.ref(), d, n, out);
        std::vector<uint8_t> got(n);
        CUSBF_CUDA_CALL(cudaMemcpy(got.data(), out, n, cudaMemcpyDeviceToHost));
        CHECK(got == want);
        // Inserting the first 25000 bytes through apply_word_masks gives the
        // engine's shard words.
        user_insert<K31><<<(25000 - K31::k + 1 + 255) / 256, 256>>>(g.ref(), d, 25000 - K31::k + 1);
        CUSBF_CUDA_CALL(cudaDeviceSynchronize());
        const uint64_t words = f.ref().num_blocks() * 4;
        std::vector<uint64_t> wf(words), wg(words);
        CUSBF_CUDA_CALL(cudaMemcpy(wf.data(), f.ref().blocks(), words * 8, cudaMemcpyDeviceToHost));
        CUSBF_CUDA_CALL(cudaMemcpy(wg.data(), g.ref().blocks(), words * 8, cudaMemcpyDeviceToHost));
        CHECK(wf == wg);
        uint64_t set = 0;
        for (uint64_t w : wf) set += w != 0;
        CHECK(set > 0);
        cudaFree(d);
        cudaFree(out);
    }
    {  // other alphabets and configurations run on the generic kernels
        using P = cusbf::Config<5, 4, 3, 4, 256, cusbf::ProteinAlphabet>;
        cusbf::filter<P> p(1 << 14);
        const std::string prot = "MKTAYIAKQRQISFVKSHFSRQ";
        CHECK(CUSBF_UNWRAP(p.insert_sequence(prot)) == prot.size() - 4);
        const auto hits = CUSBF_UNWRAP(p.contains_sequence(prot + "*WWWWW"));
        CHECK(hits.size() == prot.size() + 6 - 4);
        for (size_t i = 0; i < hits.size(); ++i)
            CHECK(hits[i] == (i < prot.size() - 4 ? 1 : i <= prot.size() ? 0 : hits[i]));
        using T = cusbf::Config<3, 2, 2, 4, 256, cusbf::DnaTripletAlphabet>;
        cusbf::filter<T> t(1 << 14);
        CHECK(CUSBF_UNWRAP(t.insert_sequence(std::string("ACGTTGCAAGGC"))) == 2);
        CHECK(all_ones(CUSBF_UNWRAP(t.contains_sequence(std::string("ACGTTGCAAGGC")))));
        using D = cusbf::Config<25, 22, 13, 8>;
        cusbf::filter<D> d(1 << 16);
        const std::string dna(200, 'C');
        CHECK(CUSBF_UNWRAP(d.insert_sequence(dna)) == 200 - 24);
        CHECK(all_ones(CUSBF_UNWRAP(d.contains_sequence(dna))));
    }
    std::printf("cpp api checks: %s\n", failures ? "FAILED" : "ok");
    return failures ? 1 : 0;
}
