// sbf_ragged.h -- ragged-launch helpers shared by the ragged batch engine
// (sbf_ragged.cu) and the request server (sbf_server.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "sbf_host.h"
#include "sbf_internal.h"

namespace sbf {

// Kernel parameters of one ragged launch over `len` bytes at d_seq.  With
// out_bits, query results are bit-packed 32-bit words at d_out (window i ->
// bit i % 32 of word i / 32).
TileParams ragged_params(const sbf_filter* f, bool query, const uint8_t* d_seq, uint64_t len,
                         const DevRange* d_rng, uint64_t n, const uint32_t* d_tile_rec,
                         uint8_t* d_out, unsigned int* queue, unsigned long long* counts,
                         bool out_bits = false);

// Stream launch of one ragged pass: tile records, queue reset, tile kernel.
int ragged_launch(sbf_filter* f, bool query, const TileParams& p, uint32_t ctas,
                  cudaStream_t st);

// The same pass replayed as a graph whose two kernel nodes are updated per
// launch (built on first use).
struct RaggedGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphNode_t n_rec{}, n_tile{};
};
int ragged_graph_launch(sbf_filter* f, RaggedGraph& g, bool query, const TileParams& p,
                        uint32_t ctas, cudaStream_t st);
void ragged_graph_release(RaggedGraph& g);

}  // namespace sbf
