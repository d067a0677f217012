/*
 * sbf_oracle.h -- CPU oracle (test infrastructure only; see sbf_oracle.c).
 */
#ifndef SBF_ORACLE_H
#define SBF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    SBF_ALPHABET_DNA = 0,
    SBF_ALPHABET_DNA_TRIPLET = 1,
    SBF_ALPHABET_PROTEIN = 2,
};

typedef struct {
    uint32_t k;
    uint32_t s;
    uint32_t m;
    uint32_t hashes;
    int32_t alphabet;
} sbf_oracle_config;

int sbf_oracle_alphabet_params(int alphabet, uint32_t* symbol_bits, uint32_t* symbol_width);
uint8_t sbf_oracle_encode(int alphabet, const char* p);
uint64_t sbf_oracle_hash64(uint64_t key);
uint64_t sbf_oracle_minimizer_hash64(uint64_t key);
uint32_t sbf_oracle_bit_address(uint32_t hashes, uint32_t j, uint64_t base_hash);
uint64_t sbf_oracle_num_shards(uint64_t requested_bits);

int sbf_oracle_insert(const sbf_oracle_config* cfg, const char* seq, uint64_t len,
                      uint64_t* words, uint64_t num_shards, int threads, uint64_t* kmers_out);
int sbf_oracle_contains(const sbf_oracle_config* cfg, const char* seq, uint64_t len,
                        const uint64_t* words, uint64_t num_shards, uint8_t* out, int threads);
int sbf_oracle_pack_dense(const sbf_oracle_config* cfg, const char* seq, uint64_t len,
                          uint64_t* words_out);
int sbf_oracle_insert_dense(const sbf_oracle_config* cfg, const uint64_t* packed,
                            uint64_t num_symbols, uint64_t* words, uint64_t num_shards,
                            int threads);
int sbf_oracle_contains_dense(const sbf_oracle_config* cfg, const uint64_t* packed,
                              uint64_t num_symbols, const uint64_t* words, uint64_t num_shards,
                              uint8_t* out, int threads);
int sbf_oracle_window_shards(const sbf_oracle_config* cfg, const char* seq, uint64_t len,
                             uint64_t num_shards, uint32_t* shards_out, uint8_t* valid_out);
int sbf_oracle_count_runs(const sbf_oracle_config* cfg, const char* seq, uint64_t len,
                          uint64_t num_shards, uint64_t* runs_out, uint64_t* valid_out);
int sbf_oracle_runs(const sbf_oracle_config* cfg, const char* seq, uint64_t len,
                    uint64_t num_shards, uint32_t* shard_out, uint64_t* masks_out,
                    uint64_t capacity, uint64_t* n_out);

#ifdef __cplusplus
}
#endif

#endif
