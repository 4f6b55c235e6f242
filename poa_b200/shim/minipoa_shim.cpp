// minipoa_shim.cpp - the drop-in for minipoa's poa() (include/align.h:15,
// src/align.cpp:1353-1737): the same signature, the DP, backtrack and path
// on the GPU through the C ABI (poa_align). Compiled against minipoa's own
// headers (graph.h, node.h, result.h, parameter.h, mem_alloc_utils.h,
// sequence.h) and linked into minipoa in place of its poa(); everything
// else in minipoa (main, alignment() with its -S sub-windows, add_path,
// topsort, output) stays as it is. It is not part of libpoa_b200.so, which
// needs no minipoa header.
//
// Per call it flattens the graph (node_t vectors -> poa_graph_view CSR
// arrays) and hands the query, already encoded by alignment()
// (src/align.cpp:1742-1745), to poa_align. One context per host thread:
// alignment() calls poa() from OpenMP threads under -S -t N
// (src/align.cpp:1800-1809). Status codes map to minipoa's own exits:
// a backtrack that leaves the band exit(0)s (src/align.cpp:1584-1588), any
// other failure prints " backtrack error" and exit(1)s (src/align.cpp:
// 1730-1731). With POA_SHIM_STATS set in the environment the number of
// GPU alignments is printed to stderr at exit.
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <vector>

#include "graph.h"
#include "mem_alloc_utils.h"
#include "poa_b200.h"
#include "result.h"
#include "sequence.h"

namespace {

std::atomic<long> g_calls(0);

struct ThreadCtx {
    poa_ctx* ctx = nullptr;
    ~ThreadCtx() {
        if (ctx) poa_destroy(ctx);
    }
};

void report() {
    if (std::getenv("POA_SHIM_STATS")) std::fprintf(stderr, "poa_shim: %ld poa() calls on the GPU\n", g_calls.load());
}

poa_ctx* context_for(const para_t* para) {
    static thread_local ThreadCtx tc;
    if (!tc.ctx) {
        poa_params p;
        poa_params_init(&p);
        p.match = para->match;
        p.mismatch = para->mismatch;
        p.gap_open = para->gap_open1;
        p.gap_ext = para->gap_ext1;
        p.band_b = para->b;
        p.band_f = para->f;
        p.ab_band = para->ab_band;
        tc.ctx = poa_create(0, &p);
        if (!tc.ctx) {
            std::cerr << "poa_shim: no GPU context" << "\n";
            std::exit(1);
        }
        static std::atomic<bool> once(false);
        if (!once.exchange(true)) std::atexit(report);
    }
    return tc.ctx;
}

}  // namespace

std::vector<res_t> poa(const para_t* para, const graph* DAG, int beg_id, int end_id, int qid, const char* qseq,
                       int qlen, aligned_buff_t* mpool, bool ab_band) {
    (void)qid;
    (void)mpool;  // the device context owns the DP memory
    poa_ctx* ctx = context_for(para);
    const int n = (int)DAG->node.size();
    std::vector<uint8_t> base(n);
    std::vector<int32_t> rank(n), par(n), ind(n), al(5 * (size_t)n), in_ptr(n + 1, 0), out_ptr(n + 1, 0);
    std::vector<int32_t> in_id, in_w, out_id;
    for (int i = 0; i < n; i++) {
        const node_t& v = DAG->node[i];
        base[i] = (uint8_t)v.base;
        rank[i] = v.rank;
        par[i] = v.par_id;
        ind[i] = v.ind;
        for (int k = 0; k < 5; k++) al[5 * (size_t)i + k] = v.aligned_node[k];
        in_id.insert(in_id.end(), v.in.begin(), v.in.end());
        in_w.insert(in_w.end(), v.in_weight.begin(), v.in_weight.end());
        out_id.insert(out_id.end(), v.out.begin(), v.out.end());
        in_ptr[i + 1] = (int32_t)in_id.size();
        out_ptr[i + 1] = (int32_t)out_id.size();
    }
    std::vector<int32_t> r2i(DAG->rank.begin(), DAG->rank.end());
    std::vector<int32_t> hlen(DAG->hlen.begin(), DAG->hlen.end()), tlen(DAG->tlen.begin(), DAG->tlen.end());
    poa_graph_view gv = {n, base.data(), rank.data(), par.data(), ind.data(), al.data(),
                         in_ptr.data(), in_id.data(), in_w.data(), out_ptr.data(), out_id.data(),
                         (int32_t)r2i.size(), r2i.data(),
                         hlen.empty() ? nullptr : hlen.data(), tlen.empty() ? nullptr : tlen.data()};
    // the query arrives encoded; minipoa maps it through char26_table once more (src/align.cpp:1364-1366)
    std::vector<uint8_t> q((size_t)qlen);
    for (int j = 0; j < qlen; j++) q[j] = (uint8_t)char26_table[(uint8_t)qseq[j]];
    std::vector<poa_res> out((size_t)n + qlen + 8);
    int32_t len = 0, score = 0;
    const int st = poa_align(ctx, &gv, beg_id, end_id, q.data(), qlen, ab_band ? 1 : 0, out.data(),
                             (int32_t)out.size(), &len, &score);
    if (st == POA_BAND_ESCAPE) std::exit(0);
    if (st != POA_OK) {
        std::cerr << " backtrack error" << "\n";
        std::exit(1);
    }
    g_calls++;
    std::vector<res_t> res;
    res.reserve(len);
    for (int k = 0; k < len; k++) res.emplace_back(res_t(out[k].from, out[k].base, out[k].aligned_id));
    return res;
}
