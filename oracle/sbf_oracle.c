/*
 * sbf_oracle.c -- CPU oracle for the Super Bloom insert/query path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA engine in
 * cusbf_b200/ is compared against; it is never linked into the product
 * library and the product never calls it.  Only tests/, the smoke check in
 * __graft_entry__.py and the CPU-baseline leg of bench.py load it.
 *
 * It restates, deliberately literally (one k-mer at a time, every m-mer and
 * s-mer hashed from scratch), the semantics of the reference cuSBF headers:
 *
 *   encode            include/cusbf/Alphabet.cuh:132-141 (DNA), :150-173
 *                     (DNA triplet), :189-217 (protein)
 *   k-mer windows     include/cusbf/detail/sequence_kmer.cuh:27-31, :75-82,
 *                     :93-102
 *   minimizer hash    include/cusbf/detail/sequence_kmer.cuh:41-51,
 *                     include/cusbf/hashutil.cuh:207-209,
 *                     include/cusbf/detail/filter_common.cuh:119-134
 *   s-mer hash        include/cusbf/detail/sequence_kmer.cuh:55-60,
 *                     include/cusbf/hashutil.cuh:192-196
 *   bit addressing    include/cusbf/detail/filter_impl.cuh:19-77,
 *                     salts include/cusbf/detail/filter_common.cuh:30-94
 *   shard selection   include/cusbf/filter_ref.cuh:52-55 with the uint32_t
 *                     truncation of include/cusbf/detail/kernels.cuh:82-83,
 *                     :149-150
 *   insert            include/cusbf/detail/kernels.cuh:107-172 (the warp
 *                     segmented OR is order independent, so a plain OR per
 *                     k-mer gives the same words)
 *   query             include/cusbf/detail/kernels.cuh:40-99,
 *                     include/cusbf/filter_ref.cuh:70-87
 *   dense packing     include/cusbf/dense_packed.hpp:36-50,
 *                     include/cusbf/detail/dense_packed.cuh:56-149
 *   shard count       include/cusbf/filter.cuh:108-118
 *
 * Pinning: tests/test_oracle.py checks this file against the reference's
 * own known-answer tests (tests/test_bloom_filter.cu of the reference) and
 * against golden vectors in tests/golden/ produced by oracle/_ref, a build of
 * the reference's own host-callable primitives (see oracle/ref_cpu.cu).
 */
#include "sbf_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* Alphabets                                                          */
/* ------------------------------------------------------------------ */

static inline uint8_t enc_dna_byte(uint8_t byte) {
    const uint8_t upper = byte & 0xDFu;
    const int valid = upper == 'A' || upper == 'C' || upper == 'G' || upper == 'T';
    return valid ? (uint8_t)((byte >> 1) & 3u) : 0xFFu;
}

static inline uint8_t enc_symbol(int alphabet, const char* p) {
    switch (alphabet) {
        case SBF_ALPHABET_DNA:
            return enc_dna_byte((uint8_t)p[0]);
        case SBF_ALPHABET_DNA_TRIPLET: {
            const uint8_t a = enc_dna_byte((uint8_t)p[0]);
            const uint8_t b = enc_dna_byte((uint8_t)p[1]);
            const uint8_t c = enc_dna_byte((uint8_t)p[2]);
            if (a == 0xFF || b == 0xFF || c == 0xFF) return 0xFFu;
            return (uint8_t)((a << 4) | (b << 2) | c);
        }
        case SBF_ALPHABET_PROTEIN: {
            const uint8_t upper = ((uint8_t)p[0]) & 0xDFu;
            const uint8_t idx = (uint8_t)(upper - 'A');
            return idx < 26 ? idx : 0xFFu;
        }
        default:
            return 0xFFu;
    }
}

int sbf_oracle_alphabet_params(int alphabet, uint32_t* symbol_bits, uint32_t* symbol_width) {
    switch (alphabet) {
        case SBF_ALPHABET_DNA:
            *symbol_bits = 2;
            *symbol_width = 1;
            return 0;
        case SBF_ALPHABET_DNA_TRIPLET:
            *symbol_bits = 6;
            *symbol_width = 3;
            return 0;
        case SBF_ALPHABET_PROTEIN:
            *symbol_bits = 5;
            *symbol_width = 1;
            return 0;
        default:
            return -1;
    }
}

uint8_t sbf_oracle_encode(int alphabet, const char* p) { return enc_symbol(alphabet, p); }

/* ------------------------------------------------------------------ */
/* Hashes and bit addressing                                          */
/* ------------------------------------------------------------------ */

static const uint64_t kSalts[16] = {
    0x9E3779B97F4A7C15ULL, 0xC2B2AE3D27D4EB4FULL, 0x165667B19E3779F9ULL, 0x85EBCA77C2B2AE63ULL,
    0x27D4EB2F165667C5ULL, 0x94D049BB133111EFULL, 0xBF58476D1CE4E5B9ULL, 0xD6E8FEB86659FD93ULL,
    0xA0761D6478BD642FULL, 0xE7037ED1A0B428DBULL, 0x8EBC6AF09C88C6E3ULL, 0x589965CC75374CC3ULL,
    0x1D8E4E27C47D124FULL, 0xEB449C93FBBEA6B5ULL, 0xDB4F0B9175AE2165ULL, 0xBBE056FDADE14B91ULL,
};

uint64_t sbf_oracle_hash64(uint64_t key) {
    key *= 0x9e3779b97f4a7c15ULL;
    key ^= key >> 33;
    return key;
}

uint64_t sbf_oracle_minimizer_hash64(uint64_t key) { return key * 0x9E3779B97F4A7C15ULL; }

static inline uint64_t window_mask(uint32_t len, uint32_t symbol_bits) {
    const uint32_t bits = len * symbol_bits;
    return bits >= 64 ? ~0ULL : ((1ULL << bits) - 1);
}

static inline uint64_t extract_sub(uint64_t packed, uint32_t start, uint32_t len, uint32_t k,
                                   uint32_t symbol_bits) {
    return (packed >> (symbol_bits * (k - (start + len)))) & window_mask(len, symbol_bits);
}

uint32_t sbf_oracle_bit_address(uint32_t hashes, uint32_t j, uint64_t base_hash) {
    const uint64_t slice = 64 / hashes;
    if (slice >= 6) {
        return (uint32_t)((base_hash >> (slice * j)) & 63u);
    }
    return (uint32_t)((base_hash * kSalts[j]) >> 58);
}

uint64_t sbf_oracle_num_shards(uint64_t requested_bits) {
    uint64_t blocks = (requested_bits + 255) / 256;
    if (blocks < 1) blocks = 1;
    uint64_t p = 1;
    while (p < blocks) p <<= 1;
    return p;
}

/* ------------------------------------------------------------------ */
/* Per-window evaluation                                              */
/* ------------------------------------------------------------------ */

typedef struct {
    uint32_t k, s, m, h;
    uint32_t bits, width;
    int alphabet;
} cfg_t;

static int make_cfg(const sbf_oracle_config* c, cfg_t* out) {
    out->k = c->k;
    out->s = c->s;
    out->m = c->m;
    out->h = c->hashes;
    out->alphabet = c->alphabet;
    if (sbf_oracle_alphabet_params(c->alphabet, &out->bits, &out->width) != 0) return -1;
    if (c->k == 0 || c->m == 0 || c->s == 0 || c->m > c->k || c->s > c->k) return -1;
    if (c->k * out->bits > 64) return -1;
    if (c->hashes == 0 || c->hashes > 16 || c->hashes % 4 != 0) return -1;
    return 0;
}

/* Evaluates window `i` given the encoded symbols.  Returns 0 when the window
 * holds an invalid symbol; otherwise fills shard and the four word masks. */
static int eval_window(const cfg_t* c, const uint8_t* sym, uint64_t i, uint64_t num_shards,
                       int dense, uint32_t* shard_out, uint64_t masks[4]) {
    uint64_t packed = 0;
    const uint64_t smask = (1ULL << c->bits) - 1;
    for (uint32_t j = 0; j < c->k; ++j) {
        const uint8_t e = sym[i + j];
        if (!dense && e == 0xFF) return 0;
        packed = (packed << c->bits) | (e & smask);
    }
    uint64_t minh = ~0ULL;
    for (uint32_t o = 0; o + c->m <= c->k; ++o) {
        const uint64_t mm = extract_sub(packed, o, c->m, c->k, c->bits);
        const uint64_t hh = sbf_oracle_minimizer_hash64(mm);
        if (hh < minh) minh = hh;
    }
    *shard_out = (uint32_t)(minh & (num_shards - 1));
    masks[0] = masks[1] = masks[2] = masks[3] = 0;
    for (uint32_t o = 0; o + c->s <= c->k; ++o) {
        const uint64_t sm = extract_sub(packed, o, c->s, c->k, c->bits);
        const uint64_t hs = sbf_oracle_hash64(sm);
        for (uint32_t j = 0; j < c->h; ++j) {
            masks[j % 4] |= 1ULL << sbf_oracle_bit_address(c->h, j, hs);
        }
    }
    return 1;
}

static uint8_t* encode_all(const cfg_t* c, const char* seq, uint64_t len, uint64_t* n_sym) {
    const uint64_t n = len / c->width;
    *n_sym = n;
    uint8_t* sym = (uint8_t*)malloc(n ? n : 1);
    if (!sym) return NULL;
    for (uint64_t t = 0; t < n; ++t) sym[t] = enc_symbol(c->alphabet, seq + t * c->width);
    return sym;
}

static uint8_t* decode_dense(const cfg_t* c, const uint64_t* words, uint64_t num_symbols) {
    const uint64_t per_word = 64 / c->bits;
    const uint64_t smask = (1ULL << c->bits) - 1;
    uint8_t* sym = (uint8_t*)malloc(num_symbols ? num_symbols : 1);
    if (!sym) return NULL;
    for (uint64_t t = 0; t < num_symbols; ++t) {
        sym[t] = (uint8_t)((words[t / per_word] >> ((t % per_word) * c->bits)) & smask);
    }
    return sym;
}

/* ------------------------------------------------------------------ */
/* Threaded drivers                                                   */
/* ------------------------------------------------------------------ */

typedef struct {
    const cfg_t* c;
    const uint8_t* sym;
    uint64_t begin, end;
    uint64_t num_shards;
    uint64_t* words;      /* insert target (atomic OR) */
    const uint64_t* ro;   /* query source */
    uint8_t* out;         /* query output */
    int dense;
    uint64_t runs;        /* run counter (count_runs) */
    uint32_t first_shard; /* count_runs: shard of the first valid window, or ~0 */
    uint32_t last_shard;
    int first_valid, last_valid;
} job_t;

static void* insert_job(void* arg) {
    job_t* j = (job_t*)arg;
    uint64_t masks[4];
    uint32_t shard;
    for (uint64_t i = j->begin; i < j->end; ++i) {
        if (!eval_window(j->c, j->sym, i, j->num_shards, j->dense, &shard, masks)) continue;
        uint64_t* w = j->words + (uint64_t)shard * 4;
        for (int q = 0; q < 4; ++q) {
            if (masks[q]) __atomic_fetch_or(&w[q], masks[q], __ATOMIC_RELAXED);
        }
    }
    return NULL;
}

static void* query_job(void* arg) {
    job_t* j = (job_t*)arg;
    uint64_t masks[4];
    uint32_t shard;
    for (uint64_t i = j->begin; i < j->end; ++i) {
        if (!eval_window(j->c, j->sym, i, j->num_shards, j->dense, &shard, masks)) {
            j->out[i] = 0;
            continue;
        }
        const uint64_t* w = j->ro + (uint64_t)shard * 4;
        int present = 1;
        for (int q = 0; q < 4; ++q) present &= (w[q] & masks[q]) == masks[q];
        j->out[i] = (uint8_t)present;
    }
    return NULL;
}

static void run_jobs(void* (*fn)(void*), job_t* base, uint64_t n_windows, int threads) {
    if (threads < 1) threads = 1;
    if ((uint64_t)threads > n_windows) threads = n_windows ? (int)n_windows : 1;
    pthread_t* tids = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
    job_t* jobs = (job_t*)calloc((size_t)threads, sizeof(job_t));
    const uint64_t per = (n_windows + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        jobs[t] = *base;
        jobs[t].begin = (uint64_t)t * per;
        jobs[t].end = jobs[t].begin + per < n_windows ? jobs[t].begin + per : n_windows;
        if (jobs[t].begin > n_windows) jobs[t].begin = n_windows;
    }
    if (threads == 1) {
        fn(&jobs[0]);
    } else {
        for (int t = 0; t < threads; ++t) pthread_create(&tids[t], NULL, fn, &jobs[t]);
        for (int t = 0; t < threads; ++t) pthread_join(tids[t], NULL);
    }
    *base = jobs[threads - 1];
    free(tids);
    free(jobs);
}

static uint64_t windows_of(const cfg_t* c, uint64_t n_sym) {
    return n_sym < c->k ? 0 : n_sym - c->k + 1;
}

int sbf_oracle_insert(const sbf_oracle_config* cfg, const char* seq, uint64_t len,
                      uint64_t* words, uint64_t num_shards, int threads, uint64_t* kmers_out) {
    cfg_t c;
    if (make_cfg(cfg, &c) != 0) return -1;
    uint64_t n_sym = 0;
    uint8_t* sym = encode_all(&c, seq, len, &n_sym);
    if (!sym) return -2;
    const uint64_t n = windows_of(&c, n_sym);
    job_t base = {0};
    base.c = &c;
    base.sym = sym;
    base.num_shards = num_shards;
    base.words = words;
    if (n) run_jobs(insert_job, &base, n, threads);
    free(sym);
    if (kmers_out) *kmers_out = n;
    return 0;
}

int sbf_oracle_contains(const sbf_oracle_config* cfg, const char* seq, uint64_t len,
                        const uint64_t* words, uint64_t num_shards, uint8_t* out, int threads) {
    cfg_t c;
    if (make_cfg(cfg, &c) != 0) return -1;
    uint64_t n_sym = 0;
    uint8_t* sym = encode_all(&c, seq, len, &n_sym);
    if (!sym) return -2;
    const uint64_t n = windows_of(&c, n_sym);
    job_t base = {0};
    base.c = &c;
    base.sym = sym;
    base.num_shards = num_shards;
    base.ro = words;
    base.out = out;
    if (n) run_jobs(query_job, &base, n, threads);
    free(sym);
    return 0;
}

int sbf_oracle_pack_dense(const sbf_oracle_config* cfg, const char* seq, uint64_t len,
                          uint64_t* words_out) {
    cfg_t c;
    if (make_cfg(cfg, &c) != 0) return -1;
    const uint64_t n = len / c.width;
    const uint64_t per_word = 64 / c.bits;
    const uint64_t n_words = (n + per_word - 1) / per_word;
    const uint64_t smask = (1ULL << c.bits) - 1;
    memset(words_out, 0, n_words * sizeof(uint64_t));
    for (uint64_t t = 0; t < n; ++t) {
        const uint8_t e = enc_symbol(c.alphabet, seq + t * c.width);
        words_out[t / per_word] |= (uint64_t)(e & smask) << ((t % per_word) * c.bits);
    }
    return 0;
}

int sbf_oracle_insert_dense(const sbf_oracle_config* cfg, const uint64_t* packed,
                            uint64_t num_symbols, uint64_t* words, uint64_t num_shards,
                            int threads) {
    cfg_t c;
    if (make_cfg(cfg, &c) != 0) return -1;
    uint8_t* sym = decode_dense(&c, packed, num_symbols);
    if (!sym) return -2;
    const uint64_t n = windows_of(&c, num_symbols);
    job_t base = {0};
    base.c = &c;
    base.sym = sym;
    base.num_shards = num_shards;
    base.words = words;
    base.dense = 1;
    if (n) run_jobs(insert_job, &base, n, threads);
    free(sym);
    return 0;
}

int sbf_oracle_contains_dense(const sbf_oracle_config* cfg, const uint64_t* packed,
                              uint64_t num_symbols, const uint64_t* words, uint64_t num_shards,
                              uint8_t* out, int threads) {
    cfg_t c;
    if (make_cfg(cfg, &c) != 0) return -1;
    uint8_t* sym = decode_dense(&c, packed, num_symbols);
    if (!sym) return -2;
    const uint64_t n = windows_of(&c, num_symbols);
    job_t base = {0};
    base.c = &c;
    base.sym = sym;
    base.num_shards = num_shards;
    base.ro = words;
    base.out = out;
    base.dense = 1;
    if (n) run_jobs(query_job, &base, n, threads);
    free(sym);
    return 0;
}

int sbf_oracle_window_shards(const sbf_oracle_config* cfg, const char* seq, uint64_t len,
                             uint64_t num_shards, uint32_t* shards_out, uint8_t* valid_out) {
    cfg_t c;
    if (make_cfg(cfg, &c) != 0) return -1;
    uint64_t n_sym = 0;
    uint8_t* sym = encode_all(&c, seq, len, &n_sym);
    if (!sym) return -2;
    const uint64_t n = windows_of(&c, n_sym);
    uint64_t masks[4];
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t shard = 0;
        valid_out[i] = (uint8_t)eval_window(&c, sym, i, num_shards, 0, &shard, masks);
        shards_out[i] = valid_out[i] ? shard : 0;
    }
    free(sym);
    return 0;
}

int sbf_oracle_count_runs(const sbf_oracle_config* cfg, const char* seq, uint64_t len,
                          uint64_t num_shards, uint64_t* runs_out, uint64_t* valid_out) {
    /* A super-k-mer run is a maximal stretch of consecutive valid windows
     * that select the same shard. */
    cfg_t c;
    if (make_cfg(cfg, &c) != 0) return -1;
    uint64_t n_sym = 0;
    uint8_t* sym = encode_all(&c, seq, len, &n_sym);
    if (!sym) return -2;
    const uint64_t n = windows_of(&c, n_sym);
    uint64_t runs = 0, valid = 0, masks[4];
    int prev_valid = 0;
    uint32_t prev_shard = 0;
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t shard = 0;
        const int v = eval_window(&c, sym, i, num_shards, 0, &shard, masks);
        if (v) {
            ++valid;
            if (!prev_valid || shard != prev_shard) ++runs;
        }
        prev_valid = v;
        prev_shard = shard;
    }
    free(sym);
    *runs_out = runs;
    if (valid_out) *valid_out = valid;
    return 0;
}

int sbf_oracle_runs(const sbf_oracle_config* cfg, const char* seq, uint64_t len,
                    uint64_t num_shards, uint32_t* shard_out, uint64_t* masks_out,
                    uint64_t capacity, uint64_t* n_out) {
    /* The super-k-mer run records of a sequence: for every maximal stretch of
     * consecutive valid windows with one shard, the shard and the OR of the
     * windows' four word masks (what one insert of the stretch ORs into the
     * shard; detail/kernels.cuh:107-172 merges windows the same way).  The
     * OR of all records into an empty filter equals sbf_oracle_insert. */
    cfg_t c;
    if (make_cfg(cfg, &c) != 0) return -1;
    uint64_t n_sym = 0;
    uint8_t* sym = encode_all(&c, seq, len, &n_sym);
    if (!sym) return -2;
    const uint64_t n = windows_of(&c, n_sym);
    uint64_t runs = 0, masks[4], acc[4] = {0, 0, 0, 0};
    int prev_valid = 0, rc = 0;
    uint32_t prev_shard = 0;
    for (uint64_t i = 0; i <= n; ++i) {
        uint32_t shard = 0;
        const int v = i < n ? eval_window(&c, sym, i, num_shards, 0, &shard, masks) : 0;
        const int cont = v && prev_valid && shard == prev_shard;
        if (prev_valid && !cont) {
            if (runs >= capacity) {
                rc = -3;
                break;
            }
            shard_out[runs] = prev_shard;
            for (int w = 0; w < 4; ++w) masks_out[4 * runs + w] = acc[w];
            ++runs;
        }
        if (v) {
            for (int w = 0; w < 4; ++w) acc[w] = (cont ? acc[w] : 0) | masks[w];
        }
        prev_valid = v;
        prev_shard = shard;
    }
    free(sym);
    *n_out = runs;
    return rc;
}
