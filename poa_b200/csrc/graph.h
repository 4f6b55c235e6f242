// graph.h - the POA graph on the host, with minipoa's semantics
// (include/graph.h:9-31, include/node.h:5-68, src/graph.cpp). The CUDA DP
// reads it through a WinView built by WindowBuilder; the batched engine keeps
// its own device-resident graph (batch.cu) with the same rules.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "dp_job.h"

namespace pb {

// One element of an alignment path, include/result.h:3-12: from >= 0 reuses
// node `from`; from < 0 creates a node with `base`, aligned to `aligned_id`
// (a mismatch) when aligned_id >= 0.
struct Res {
    int32_t from;
    uint8_t base;
    int32_t aligned_id;
};

struct Node {
    int32_t id, rank, par_id, ind;
    uint8_t base;
    int32_t aligned[5];
    std::vector<int32_t> in, in_w, out, out_w;
    std::vector<int32_t> ids, idp;  // read ords through the node (MSA rows / GFA paths)
};

class Graph {
  public:
    Graph();                                            // source 0 and sink 1, src/graph.cpp:129-135
    int add_node(uint8_t base);
    void add_adj(int seq_id, int from, int to, int cur_pos);          // src/graph.cpp:13-20
    void add_path(int seq_id, const std::vector<Res>& res, int sink_id);  // src/graph.cpp:170-235
    void topsort(bool with_lens, bool seeding, int op);               // src/graph.cpp:21-128
    void build_consensus(bool need_coverages);                        // src/graph.cpp:294-351
    std::vector<std::string> msa_rows(int nseq) const;                // src/graph.cpp:237-251
    // GFA text, src/graph.cpp:358-434; read_len / names by input index,
    // rid_to_ord maps them to the read ord used in the graph.
    void gfa_text(const std::vector<int32_t>& read_len, const std::vector<std::string>& names,
                  const std::vector<int32_t>& rid_to_ord, std::string& out) const;

    std::vector<Node> node;
    std::vector<int32_t> rank;        // rank -> node id
    std::vector<int32_t> hlen, tlen;  // by rank; resized like std::vector::resize in the reference
    bool is_topsorted = false;
    std::string cons;                 // ASCII consensus
    std::vector<int32_t> cons_pos_to_id, coverages;
};

// Flat window view of ranks [rank(beg_id), rank(end_id)] in host memory.
struct HostWindow {
    int32_t n = 0, beg_i = 0, end_i = 0;
    std::vector<int32_t> row_node;  // node id of each row
    std::vector<int32_t> in_ptr, in_row, in_w;
    std::vector<uint8_t> in_base, base;
    std::vector<int32_t> ind, hq, hq_loc, tq, out_ptr, out_row;
    int32_t max_indeg = 0;
};

// Build the window view. with_lens: the graph carries hlen/tlen (f > 0).
void build_window(const Graph& g, int beg_id, int end_id, bool with_lens, HostWindow& w);

// Convert backtrack moves (in backtrack order) into a forward path,
// src/align.cpp:1606-1620 (match / mismatch emission) and :1672-1682 (insert).
void moves_to_path(const Graph& g, const HostWindow& w, const int32_t* moves, int n, std::vector<Res>& out);

// ASCII -> 0..4 (src/sequence.cpp:6-23); codes 0..3 map to themselves.
uint8_t nt4(uint8_t c);
extern const char kNt256[5];

}  // namespace pb
