// driver.cpp - the reference's read loop and alignment() dispatch over a DP
// engine. The DP itself (every poa() call) runs in the engine; this file
// keeps the host-side control flow of src/main.cpp:84-126 and
// src/align.cpp:1741-1828.
#include "driver.h"

#include <numeric>
#include <unordered_map>

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

int32_t load_gfa(const Params& p, const std::string& text, Graph& g, std::vector<std::string>& path_names,
                 std::string& err) {
    std::unordered_map<std::string, int> seg;  // segment name -> index
    std::vector<int32_t> seg_first, seg_last;  // its first / last node id
    size_t pos = 0;
    while (pos < text.size()) {
        size_t eol = text.find('\n', pos);
        if (eol == std::string::npos) eol = text.size();
        std::string line = text.substr(pos, eol - pos);
        pos = eol + 1;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.size() < 3 || line[1] != '\t') continue;
        if (line[0] != 'S' && line[0] != 'P') continue;
        // the first two tab-separated fields after the record type
        std::vector<std::string> f;
        size_t a = 2;
        while (f.size() < 2) {
            size_t t = line.find('\t', a);
            if (t == std::string::npos) { f.push_back(line.substr(a)); break; }
            f.push_back(line.substr(a, t - a));
            a = t + 1;
        }
        if (f.size() < 2) {
            err = line[0] == 'S' ? "no seq in GFA segment line (" + f[0] + ")" : "no path in GFA path line (" + f[0] + ")";
            return ST_BAD_ARG;
        }
        if (line[0] == 'S') {  // gfa_parse_S, src/handle_input.cpp:78-128
            if (seg.count(f[0])) { err = "duplicated segment " + f[0]; return ST_BAD_ARG; }
            if (f[1].empty()) { err = "empty segment " + f[0]; return ST_BAD_ARG; }
            seg[f[0]] = (int)seg_first.size();
            int first = -1, last = -1;
            for (char c : f[1]) {
                last = g.add_node(nt4((uint8_t)c));
                if (first < 0) first = last;
            }
            seg_first.push_back(first);
            seg_last.push_back(last);
            continue;
        }
        // gfa_parse_P, src/handle_input.cpp:129-246: "name+,name+,..." (or all '-')
        const int pid = (int)path_names.size();
        const std::string& walk = f[1];
        int is_rc = -1, last_id = 0, next_id = 1, cur_pos = 0;
        size_t start = 0;
        for (size_t k = 0; k < walk.size(); k++) {
            const char c = walk[k];
            if (c != '+' && c != '-') continue;
            const std::string name = walk.substr(start, k - start);
            const bool rc = c == '-';
            if ((rc && is_rc == 0) || (!rc && is_rc == 1)) {
                err = "path has both '+' and '-' segments (" + f[0] + ")";
                return ST_BAD_ARG;
            }
            is_rc = rc ? 1 : 0;
            auto it = seg.find(name);
            if (it == seg.end()) { err = "segment " + name + " does not exist"; return ST_BAD_ARG; }
            const int in_id = seg_first[it->second], out_id = seg_last[it->second];
            if (!rc) {
                g.add_adj(pid, last_id, in_id, cur_pos++);
                for (int i = 0; i < out_id - in_id; i++) g.add_adj(pid, in_id + i, in_id + i + 1, cur_pos++);
                last_id = out_id;
            } else {
                g.add_adj(pid, out_id, next_id, cur_pos++);
                for (int i = 0; i < out_id - in_id; i++) g.add_adj(pid, in_id + i, in_id + i + 1, cur_pos++);
                next_id = in_id;
            }
            start = k + 2;  // past the sign and the separator
        }
        if (is_rc != 0) g.add_adj(pid, 0, next_id, cur_pos++);  // also when no segment was signed, as in the reference
        else g.add_adj(pid, last_id, 1, cur_pos++);
        path_names.push_back(f[0]);
    }
    g.topsort(p.f > 0, p.enable_seeding != 0, 0);
    return ST_OK;
}

int32_t run_reads(const Params& p, const std::vector<std::string>& reads,
                  const std::vector<std::string>& read_headers, DpEngine& eng, std::string& text,
                  std::vector<int32_t>* scores, RunStats* stats, const std::string* gfa) {
    (void)stats;
    Graph g;
    // an existing graph's paths come first, as reads without bases (src/main.cpp:86-96)
    std::vector<std::string> seqs, headers;
    int exist = 0;
    if (gfa) {
        std::vector<std::string> names;
        std::string err;
        const int32_t st = load_gfa(p, *gfa, g, names, err);
        if (st != ST_OK) { text = err; return st; }
        exist = (int)names.size();
        seqs.assign(exist, std::string());
        for (const std::string& nm : names) headers.push_back(nm + " ");
    }
    seqs.insert(seqs.end(), reads.begin(), reads.end());
    for (size_t i = 0; i < reads.size(); i++) headers.push_back(i < read_headers.size() ? read_headers[i] : "");
    const int nseq = (int)seqs.size();
    std::vector<int32_t> ord(nseq);
    std::iota(ord.begin(), ord.end(), 0);
    std::vector<int32_t> rid_to_ord = ord;
    Seeder* seeder = nullptr;
    Seeder sd;
    if (p.enable_seeding || p.progressive) {
        sd.init(p, seqs);
        seeder = &sd;
        if (p.progressive && !gfa) {  // no guide tree when extending a graph (src/main.cpp:101)
            sd.guide_tree(p);
            ord = sd.ord;
            rid_to_ord = sd.rid_to_ord;
        }
    }
    std::vector<Res> res;
    std::vector<uint8_t> q;
    for (int i = exist; i < nseq; i++) {
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
