// driver.cpp - the reference's read loop and alignment() dispatch over a DP
// engine. The DP itself (every poa() call) runs in the engine; this file
// keeps the host-side control flow of src/main.cpp:84-126 and
// src/align.cpp:1741-1828.
#include "driver.h"

#include <numeric>

#include "seeding.h"

namespace pb {

void normalize_params(Params& p) {
    // src/handle_input.cpp:47 negates para->m rather than match; match keeps its sign
    if (p.mismatch > 0) p.mismatch = -p.mismatch;
    if (p.gap_open1 > 0) p.gap_open1 = -p.gap_open1;
    if (p.gap_ext1 > 0) p.gap_ext1 = -p.gap_ext1;
}

Scoring scoring_of(const Params& p) {
    Scoring s;
    s.match = p.match;
    s.mismatch = p.mismatch;
    s.e1 = p.gap_ext1;
    s.o1 = p.gap_open1 + p.gap_ext1;
    return s;
}

namespace {

int32_t run_one(const Params& p, const Graph& g, DpEngine& eng, int beg_id, int end_id, const uint8_t* q,
                int qlen, int ab_band, std::vector<Res>& out, std::vector<int32_t>* scores) {
    HostWindow w;
    build_window(g, beg_id, end_id, p.f > 0, w);
    std::vector<AlignOut> outs;
    eng.align_many({&w}, {q}, {qlen}, {ab_band}, p, outs);
    if (outs[0].status != ST_OK) return outs[0].status;
    if (scores) scores->push_back(outs[0].score);
    moves_to_path(g, w, outs[0].moves.data(), (int)outs[0].moves.size(), out);
    return ST_OK;
}

}  // namespace

int32_t alignment(const Params& p, Graph& g, Seeder* seeder, int rid, const uint8_t* q, int qlen,
                  DpEngine& eng, std::vector<Res>& res, std::vector<int32_t>* scores) {
    res.clear();
    if (g.node.size() <= 2) {  // src/align.cpp:1747-1753
        res.push_back(Res{0, 4, -1});
        for (int j = 0; j < qlen; j++) res.push_back(Res{-1, q[j], -1});
        return ST_OK;
    }
    if (!p.enable_seeding) return run_one(p, g, eng, 0, 1, q, qlen, p.ab_band, res, scores);
    if (!seeder) return ST_BAD_ARG;
    if (!g.is_topsorted) g.topsort(p.f > 0, true, 0);
    std::vector<Anchor> anchors;
    seeder->anchors_by_consensus(p, rid, qlen, g.cons, anchors);
    const int ab = 1;  // src/align.cpp:1764: sub-windows always use the adaptive band
    if (anchors.empty()) return run_one(p, g, eng, 0, 1, q, qlen, ab, res, scores);
    // src/align.cpp:1796-1823 (the -t > 1 form; the serial form :1769-1795 gives
    // the same path when every anchor spans k bases): K+1 independent sub-windows
    const int K = (int)anchors.size(), kq = p.k;
    std::vector<HostWindow> wins(K + 1);
    std::vector<const HostWindow*> wp(K + 1);
    std::vector<const uint8_t*> qp(K + 1);
    std::vector<int32_t> ql(K + 1), abv(K + 1, ab);
    for (int i = 0; i <= K; i++) {
        int beg_id = i == 0 ? 0 : g.cons_pos_to_id[(int32_t)anchors[i - 1].x];
        int end_id = i == K ? 1 : g.cons_pos_to_id[(int32_t)anchors[i].x - kq + 1];
        int end_qpos = i == K ? qlen : (int32_t)anchors[i].y - kq + 1;
        int start_qpos = i == 0 ? 0 : (int32_t)anchors[i - 1].y + 1;
        build_window(g, beg_id, end_id, p.f > 0, wins[i]);
        wp[i] = &wins[i];
        qp[i] = q + start_qpos;
        ql[i] = end_qpos - start_qpos;
        if (wins[i].n <= 0 || ql[i] < 0) return ST_DEGENERATE;  // the reference faults here (src/align.cpp:1400)
    }
    std::vector<AlignOut> outs;
    eng.align_many(wp, qp, ql, abv, p, outs);
    std::vector<Res> part;
    for (int i = 0; i <= K; i++) {
        if (outs[i].status != ST_OK) return outs[i].status;
        if (scores) scores->push_back(outs[i].score);
        moves_to_path(g, wins[i], outs[i].moves.data(), (int)outs[i].moves.size(), part);
        res.insert(res.end(), part.begin(), part.end());
        if (i < K) {
            int end_tpos = (int32_t)anchors[i].x - kq + 1;
            for (int k = 0; k < kq - 1; k++) {
                const Node& cur = g.node[g.cons_pos_to_id[end_tpos + k]];
                res.push_back(Res{cur.id, cur.base, -1});
            }
        }
    }
    return ST_OK;
}

int32_t run_reads(const Params& p, const std::vector<std::string>& seqs,
                  const std::vector<std::string>& headers, DpEngine& eng, std::string& text,
                  std::vector<int32_t>* scores, RunStats* stats) {
    (void)stats;
    const int nseq = (int)seqs.size();
    Graph g;
    std::vector<int32_t> ord(nseq);
    std::iota(ord.begin(), ord.end(), 0);
    std::vector<int32_t> rid_to_ord = ord;
    Seeder* seeder = nullptr;
    Seeder sd;
    if (p.enable_seeding || p.progressive) {
        sd.init(p, seqs);
        seeder = &sd;
        if (p.progressive) {
            sd.guide_tree(p);
            ord = sd.ord;
            rid_to_ord = sd.rid_to_ord;
        }
    }
    std::vector<Res> res;
    std::vector<uint8_t> q;
    for (int i = 0; i < nseq; i++) {
        int rid = ord[i];
        const std::string& s = seqs[rid];
        q.resize(s.size());
        for (size_t j = 0; j < s.size(); j++) q[j] = nt4((uint8_t)s[j]);
        int32_t st = alignment(p, g, seeder, rid, q.data(), (int)q.size(), eng, res, scores);
        if (st != ST_OK) return st;
        g.add_path(i, res, 1);
        g.topsort(p.f > 0, p.enable_seeding != 0, i + 1 == nseq);
    }
    text.clear();
    if (p.result == 0) {  // src/graph.cpp:352-357
        g.build_consensus(false);
        text = ">consensus sequence\n" + g.cons + "\n";
    } else if (p.result == 1) {  // src/graph.cpp:237-251
        if (!g.is_topsorted) g.topsort(p.f > 0, false, 1);
        std::vector<std::string> rows = g.msa_rows(nseq);
        for (int i = 0; i < nseq; i++) {
            if (i < (int)headers.size() && !headers[i].empty()) text += ">" + headers[i] + "\n";
            else text += ">" + std::to_string(i + 1) + "\n";
            text += rows[rid_to_ord[i]];
            text += "\n";
        }
    } else if (p.result == 2) {  // src/graph.cpp:358-434; names are the first word of each header
        std::vector<int32_t> lens(nseq);
        std::vector<std::string> names(nseq);
        for (int i = 0; i < nseq; i++) {
            lens[i] = (int32_t)seqs[i].size();
            if (i < (int)headers.size()) names[i] = headers[i].substr(0, headers[i].find(' '));
        }
        g.gfa_text(lens, names, rid_to_ord, text);
    }  // other values print nothing, as in src/main.cpp:124-126
    return ST_OK;
}

}  // namespace pb
