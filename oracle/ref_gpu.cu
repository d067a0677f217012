// ref_gpu.cu -- extern "C" handle over the UNMODIFIED reference cuSBF GPU
// filter (include/cusbf/filter.cuh of tdortman/cuSBF), compiled for sm_100a.
//
// TEST INFRASTRUCTURE ONLY (built into oracle/_ref/, never shipped).  GPU
// parity tests use it to check that the engine's filter words and query
// bytes equal the reference GPU path's on the same input, and to time the
// reference kernels beside the engine's.  It calls the reference's public
// API exactly as its benchmark does (insert_sequence_async /
// contains_sequence_async, benchmarks/benchmark_common.cuh:987-1035).
#include <cstdint>
#include <new>

#include <cusbf/filter.cuh>

namespace {
using C31 = cusbf::Config<31, 28, 16, 4>;
using C5 = cusbf::Config<5, 4, 3, 4>;
using C31H8 = cusbf::Config<31, 28, 16, 8>;
using C31H16 = cusbf::Config<31, 28, 16, 16>;
using C21 = cusbf::Config<21, 19, 11, 4>;
using C31M21 = cusbf::Config<31, 28, 21, 4>;                       // 7
using C25 = cusbf::Config<25, 22, 13, 4>;                          // 8
using CP12 = cusbf::Config<12, 10, 6, 4, 256, cusbf::ProteinAlphabet>;  // 9
using C31S30 = cusbf::Config<31, 30, 16, 4>;                       // 10
using C31S31 = cusbf::Config<31, 31, 16, 4>;                       // 11

struct Handle {
    int cfg;
    void* f;
};

// filter::ref() const does not instantiate in the reference (it converts a
// const shard pointer to a non-const one), so the shard vector is reached
// through the explicit-instantiation access rule instead.
template <typename Tag, typename Tag::type Member>
struct ShardAccess {
    friend typename Tag::type shard_member(Tag) { return Member; }
};

#define SBF_REF_SHARDS(Tag, Cfg)                                                          \
    struct Tag {                                                                          \
        using type = thrust::device_vector<cusbf::filter_block<Cfg>> cusbf::filter<Cfg>::*; \
        friend type shard_member(Tag);                                                    \
    };                                                                                    \
    template struct ShardAccess<Tag, &cusbf::filter<Cfg>::d_shards_>;                     \
    const void* shard_ptr(cusbf::filter<Cfg>& f) {                                        \
        return thrust::raw_pointer_cast((f.*shard_member(Tag{})).data());                 \
    }

SBF_REF_SHARDS(Shards31, C31)
SBF_REF_SHARDS(Shards5, C5)
SBF_REF_SHARDS(Shards31H8, C31H8)
SBF_REF_SHARDS(Shards31H16, C31H16)
SBF_REF_SHARDS(Shards21, C21)
SBF_REF_SHARDS(Shards31M21, C31M21)
SBF_REF_SHARDS(Shards25, C25)
SBF_REF_SHARDS(ShardsP12, CP12)
SBF_REF_SHARDS(Shards31S30, C31S30)
SBF_REF_SHARDS(Shards31S31, C31S31)

// Configuration ids: 0-6 as in oracle/oracle.py REF_CONFIGS; 7-9 extra
// configurations (a long minimizer, one with no specialised engine kernel,
// and a protein alphabet); 10-11 the s = 30 and s = 31 columns of the
// reference's false-positive sweep (benchmarks/fpr_fastx_sweep.cu).
template <typename Fn>
int with(Handle* h, Fn&& fn) {
    if (!h) return -1;
    switch (h->cfg) {
        case 0: return fn(*static_cast<cusbf::filter<C31>*>(h->f));
        case 1: return fn(*static_cast<cusbf::filter<C5>*>(h->f));
        case 4: return fn(*static_cast<cusbf::filter<C31H8>*>(h->f));
        case 5: return fn(*static_cast<cusbf::filter<C31H16>*>(h->f));
        case 6: return fn(*static_cast<cusbf::filter<C21>*>(h->f));
        case 7: return fn(*static_cast<cusbf::filter<C31M21>*>(h->f));
        case 8: return fn(*static_cast<cusbf::filter<C25>*>(h->f));
        case 9: return fn(*static_cast<cusbf::filter<CP12>*>(h->f));
        case 10: return fn(*static_cast<cusbf::filter<C31S30>*>(h->f));
        case 11: return fn(*static_cast<cusbf::filter<C31S31>*>(h->f));
        default: return -1;
    }
}
}  // namespace

extern "C" {

void* sbf_refgpu_create(int cfg, uint64_t bits) {
    try {
        switch (cfg) {
            case 0: return new Handle{0, new cusbf::filter<C31>(bits)};
            case 1: return new Handle{1, new cusbf::filter<C5>(bits)};
            case 4: return new Handle{4, new cusbf::filter<C31H8>(bits)};
            case 5: return new Handle{5, new cusbf::filter<C31H16>(bits)};
            case 6: return new Handle{6, new cusbf::filter<C21>(bits)};
            case 7: return new Handle{7, new cusbf::filter<C31M21>(bits)};
            case 8: return new Handle{8, new cusbf::filter<C25>(bits)};
            case 9: return new Handle{9, new cusbf::filter<CP12>(bits)};
            case 10: return new Handle{10, new cusbf::filter<C31S30>(bits)};
            case 11: return new Handle{11, new cusbf::filter<C31S31>(bits)};
            default: break;
        }
    } catch (...) {
    }
    return nullptr;
}

void sbf_refgpu_destroy(void* p) {
    auto* h = static_cast<Handle*>(p);
    if (!h) return;
    with(h, [](auto& f) {
        delete &f;
        return 0;
    });
    delete h;
}

int sbf_refgpu_clear(void* p, cudaStream_t stream) {
    return with(static_cast<Handle*>(p), [&](auto& f) { return f.clear(stream) ? 0 : 1; });
}

int sbf_refgpu_insert_async(void* p, const char* d_seq, uint64_t len, cudaStream_t stream) {
    return with(static_cast<Handle*>(p), [&](auto& f) {
        auto r = f.insert_sequence_async(cusbf::device_span<const char>{d_seq, len}, stream);
        return r ? 0 : 1;
    });
}

int sbf_refgpu_contains_async(void* p, const char* d_seq, uint64_t len, uint8_t* d_out,
                              uint64_t out_len, cudaStream_t stream) {
    return with(static_cast<Handle*>(p), [&](auto& f) {
        auto r = f.contains_sequence_async(cusbf::device_span<const char>{d_seq, len},
                                           cusbf::device_span<uint8_t>{d_out, out_len}, stream);
        return r ? 0 : 1;
    });
}

const void* sbf_refgpu_words(void* p) {
    const void* out = nullptr;
    with(static_cast<Handle*>(p), [&](auto& f) {
        out = shard_ptr(f);
        return 0;
    });
    return out;
}

uint64_t sbf_refgpu_num_shards(void* p) {
    uint64_t out = 0;
    with(static_cast<Handle*>(p), [&](auto& f) {
        out = f.num_shards();
        return 0;
    });
    return out;
}
}
