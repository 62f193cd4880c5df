// image.h — host-side packing of a component into the device program image.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/ksim_b200.h"

namespace ksim {

// Per graph (32 B): term count, parameter count, and where its term stream lies.
struct GraphDir {
    int32_t G, P, n_chunks, first_chunk;
    int64_t stream_off, stream_bytes;
};

// Per staging chunk (32 B): a run of whole terms of one graph, <= slot bytes.
struct ChunkDir {
    int64_t off;
    int32_t bytes, graph, n_terms, end_of_graph;
    int32_t pad0, pad1;
};

static_assert(sizeof(GraphDir) == 32, "GraphDir layout");
static_assert(sizeof(ChunkDir) == 32, "ChunkDir layout");

// Supported parameter-vector widths (64-bit words); images are padded up to one.
int supported_words(int needed);

struct HostImage {
    int n_graphs = 0, F = 0, n_out = 0, W = 0;
    std::vector<uint8_t> bytes;                  // [GraphDir x n_graphs][term streams]
    std::vector<GraphDir> gdir;
    std::vector<std::vector<int64_t>> term_off;  // per graph: term start offsets + end
    int64_t max_term_bytes = 0;
    int64_t n_terms = 0, n_slow_terms = 0, n_narrow_terms = 0, n_hybrid_terms = 0;
    double work_ops = 0;  // int32 operations per shot, all graphs (term_work / graph_work)
    int64_t n_columns = 0;
};

// Validate the descriptors and pack them.  Returns a ksim_status; on failure
// `err` says which graph / array is wrong.
int build_image(const ksim_graph_desc *graphs, int n_graphs, int F, HostImage &out,
                std::string &err);

// int32 operations of one shot for one term / one graph (the roofline
// numerator; see image.cpp).
double term_work(int W, uint32_t flags, const int n_cls[4], int n_hp, int n_pp, int n_ph, int nb, int sum_iter);
double graph_work(int W);

// Split every graph's term stream into chunks of whole terms of at most
// slot_bytes (an empty graph gets one empty chunk).  Returns false if a single
// term is larger than slot_bytes.
bool make_chunks(const HostImage &img, int64_t slot_bytes, std::vector<ChunkDir> &out);

// (1 - w)-adic valuation of a Z[w] element given as 4 int64 (15 for zero);
// exposed for tests.
uint32_t zw_valuation(const int64_t z[4]);

}  // namespace ksim
