// graph.cpp - host POA graph with minipoa's fusion, ordering and consensus
// rules. Every method states the reference lines whose behaviour it keeps;
// ordering details (in-list order, LIFO topological order, first-max
// tie-breaks) are kept exactly because the DP band, the backtrack tie-breaks
// and the MSA column order depend on them.
#include "graph.h"

#include <algorithm>

namespace pb {

const char kNt256[5] = {'A', 'C', 'G', 'T', 'N'};  // src/sequence.cpp:26-43

uint8_t nt4(uint8_t c) {  // src/sequence.cpp:6-23
    switch (c) {
        case 0: case 1: case 2: case 3: return c;
        case 'A': case 'a': return 0;
        case 'C': case 'c': return 1;
        case 'G': case 'g': return 2;
        case 'T': case 't': case 'U': case 'u': return 3;
        default: return 4;
    }
}

Graph::Graph() {
    add_node(4);  // source
    add_node(4);  // sink
}

int Graph::add_node(uint8_t base) {  // node_t ctor, include/node.h:16-22
    Node v;
    v.id = v.par_id = (int32_t)node.size();
    v.rank = 0;
    v.ind = 0;
    v.base = base;
    for (int k = 0; k < 5; k++) v.aligned[k] = -1;
    v.aligned[base] = v.id;
    node.push_back(std::move(v));
    return (int)node.size() - 1;
}

// include/node.h:23-61 through src/graph.cpp:13-20: repeated edges add weight,
// new edges append (in-list / out-list order is insertion order).
void Graph::add_adj(int seq_id, int from, int to, int cur_pos) {
    if (from == to) return;
    Node& f = node[from];
    bool ok = false;
    for (size_t i = 0; i < f.out.size(); i++)
        if (f.out[i] == to) { f.out_w[i]++; ok = true; break; }
    if (!ok) { f.out.push_back(to); f.out_w.push_back(1); }
    if (f.ids.empty() || f.ids.back() != seq_id) f.ids.push_back(seq_id);

    Node& t = node[to];
    t.ind++;
    ok = false;
    for (size_t i = 0; i < t.in.size(); i++)
        if (t.in[i] == from) { t.in_w[i]++; ok = true; break; }
    if (!ok) { t.in.push_back(from); t.in_w.push_back(1); }
    if (t.ids.empty() || t.ids.back() != seq_id) {
        t.ids.push_back(seq_id);
        t.idp.push_back(cur_pos);
    }
}

void Graph::add_path(int seq_id, const std::vector<Res>& res, int sink_id) {
    int anchored = -1, cur_pos = 0;
    for (const Res& r : res) {
        int cur = r.from;
        if (cur < 0) {
            if (r.aligned_id >= 0) {  // mismatch: reuse or create the aligned sibling
                int al = r.aligned_id;
                if (node[al].aligned[r.base] == -1) {
                    cur = add_node(r.base);
                    node[al].aligned[r.base] = cur;
                    node[cur].par_id = al;
                } else {
                    cur = node[al].aligned[r.base];
                }
            } else {
                cur = add_node(r.base);
            }
        }
        if (anchored != -1) add_adj(seq_id, anchored, cur, cur_pos++);
        anchored = cur;
    }
    if (sink_id != -1) add_adj(seq_id, anchored, sink_id, cur_pos);
    is_topsorted = false;
}

void Graph::topsort(bool with_lens, bool seeding, int op) {
    const int N = (int)node.size();
    std::vector<int32_t> deg(N, 0), stk;
    stk.reserve(N);
    rank.clear();
    if (op == 1) {  // src/graph.cpp:24-59: one rank per aligned group
        for (int i = 0; i < N; i++) {
            Node& v = node[i];
            v.rank = -1;
            if (v.par_id != v.id) continue;
            int s = 0;
            for (int k = 0; k < 5; k++)
                if (v.aligned[k] >= 0) s += (int)node[v.aligned[k]].in.size();
            deg[i] = s;
            if (s == 0) stk.push_back(i);
        }
        while (!stk.empty()) {
            int u = stk.back();
            stk.pop_back();
            node[u].rank = (int32_t)rank.size();
            rank.push_back(u);
            for (int k = 0; k < 5; k++) {
                int sid = node[u].aligned[k];
                if (sid < 0) continue;
                node[sid].rank = node[u].rank;
                for (int32_t o : node[sid].out) {
                    int v = node[o].par_id;
                    if (--deg[v] == 0) stk.push_back(v);
                }
            }
        }
        is_topsorted = true;
        return;
    }
    // src/graph.cpp:61-85: Kahn with a LIFO stack, zero in-degree nodes seeded in id order
    for (int i = 0; i < N; i++) {
        deg[i] = (int32_t)node[i].in.size();
        if (deg[i] == 0) stk.push_back(i);
    }
    while (!stk.empty()) {
        int u = stk.back();
        stk.pop_back();
        node[u].rank = (int32_t)rank.size();
        rank.push_back(u);
        for (int32_t v : node[u].out)
            if (--deg[v] == 0) stk.push_back(v);
    }
    is_topsorted = true;
    if (with_lens) {  // src/graph.cpp:86-123: heaviest-edge depth from source / to sink
        hlen.resize(N);
        for (size_t i = 0; i < rank.size(); i++) {
            const Node& cur = node[rank[i]];
            int wmax = -1, max_pre = -1;
            for (size_t k = 0; k < cur.in.size(); k++)
                if (cur.in_w[k] > wmax) { wmax = cur.in_w[k]; max_pre = node[cur.in[k]].rank; }
            if (max_pre != -1) hlen[cur.rank] = hlen[max_pre] + 1;
        }
        tlen.resize(N);
        tlen[node[1].rank] = 1;
        for (int i = (int)rank.size() - 1; i >= 0; i--) {
            const Node& cur = node[rank[i]];
            int wmax = -1, max_suc = -1;
            for (size_t k = 0; k < cur.out.size(); k++)
                if (cur.out_w[k] > wmax) { wmax = cur.out_w[k]; max_suc = node[cur.out[k]].rank; }
            if (max_suc != -1) tlen[cur.rank] = tlen[max_suc] + 1;
        }
    }
    if (seeding) build_consensus(false);  // src/graph.cpp:127
}

// src/graph.cpp:294-351: FIFO Kahn from the source; each node keeps the
// heaviest in-edge, ties to the larger accumulated score (first wins).
void Graph::build_consensus(bool need_coverages) {
    const int N = (int)node.size();
    std::vector<int32_t> deg(N), pre(N, 0), score(N, 0), q;
    q.reserve(N);
    for (int i = 0; i < N; i++) deg[i] = (int32_t)node[i].in.size();
    q.push_back(0);
    for (size_t h = 0; h < q.size(); h++) {
        int u = q[h];
        const Node& cur = node[u];
        if (u != 0) {
            int wmax = -1, max_pre = -1;
            for (size_t k = 0; k < cur.in.size(); k++) {
                int pr = node[cur.in[k]].id, wk = cur.in_w[k];
                if (wk > wmax || (wk == wmax && score[pr] > score[max_pre])) { wmax = wk; max_pre = pr; }
            }
            pre[u] = max_pre;
            score[u] = score[max_pre] + wmax;
        }
        if (u == 1) break;
        for (int32_t v : cur.out)
            if (--deg[v] == 0) q.push_back(v);
    }
    if (need_coverages) coverages.clear();
    cons.clear();
    cons_pos_to_id.clear();
    for (int id = pre[1]; id != 0; id = pre[id]) {
        const Node& cur = node[id];
        cons.push_back(kNt256[cur.base]);
        cons_pos_to_id.push_back(cur.id);
        if (need_coverages) {
            int in_w = 0, out_w = 0;
            for (int32_t x : cur.in_w) in_w += x;
            for (int32_t x : cur.out_w) out_w += x;
            coverages.push_back(std::max(in_w, out_w));
        }
    }
    std::reverse(cons.begin(), cons.end());
    std::reverse(cons_pos_to_id.begin(), cons_pos_to_id.end());
    if (need_coverages) std::reverse(coverages.begin(), coverages.end());
}

// src/graph.cpp:237-251 after the op==1 topsort: column = rank of the aligned
// group's parent minus one; row = read ord.
std::vector<std::string> Graph::msa_rows(int nseq) const {
    int nc = (int)rank.size() - 2;
    if (nc < 0) nc = 0;
    std::vector<std::string> rows(nseq, std::string(nc, '-'));
    for (size_t i = 2; i < node.size(); i++) {
        int rk = node[node[i].par_id].rank;
        if (rk - 1 < 0 || rk - 1 >= nc) continue;
        for (int32_t id : node[i].ids)
            if (id >= 0 && id < nseq) rows[id][rk - 1] = kNt256[node[i].base];
    }
    return rows;
}

void build_window(const Graph& g, int beg_id, int end_id, bool with_lens, HostWindow& w) {
    const int beg_i = g.node[beg_id].rank, end_i = g.node[end_id].rank;
    const int n = end_i - beg_i + 1;
    w.n = n;
    w.beg_i = beg_i;
    w.end_i = end_i;
    w.max_indeg = 0;
    if (n <= 0) return;
    w.row_node.resize(n);
    w.base.resize(n);
    w.ind.resize(n);
    w.hq.assign(n, 0);
    w.hq_loc.assign(n, 0);
    w.tq.assign(n, 0);
    w.in_ptr.assign(n + 1, 0);
    w.out_ptr.assign(n + 1, 0);
    w.in_row.clear(); w.in_w.clear(); w.in_base.clear(); w.out_row.clear();
    for (int r = 0; r < n; r++) {
        const Node& v = g.node[g.rank[beg_i + r]];
        w.row_node[r] = v.id;
        w.base[r] = v.base;
        w.ind[r] = v.ind;
        if (with_lens) {
            w.hq[r] = g.hlen[beg_i + r] - g.hlen[beg_i];
            w.hq_loc[r] = g.hlen[r] - g.hlen[beg_i];
            w.tq[r] = g.tlen[beg_i + r] - g.tlen[end_i];
        }
        int deg = 0;
        for (size_t k = 0; k < v.in.size(); k++) {
            int p = g.node[v.in[k]].rank - beg_i;
            if (p < 0) continue;  // src/align.cpp:1451-1452
            w.in_row.push_back(p);
            w.in_w.push_back(v.in_w[k]);
            w.in_base.push_back(p == 0 ? 4 : g.node[v.in[k]].base);  // src/align.cpp:1453
            deg++;
        }
        w.max_indeg = std::max(w.max_indeg, deg);
        w.in_ptr[r + 1] = (int32_t)w.in_row.size();
        for (int32_t o : v.out) {
            int s = g.node[o].rank - beg_i;
            if (s >= n) continue;  // src/align.cpp:1550-1551
            w.out_row.push_back(s);
        }
        w.out_ptr[r + 1] = (int32_t)w.out_row.size();
    }
}

void moves_to_path(const Graph& g, const HostWindow& w, const int32_t* moves, int n, std::vector<Res>& out) {
    out.clear();
    out.reserve(n);
    for (int t = n - 1; t >= 0; t--) {
        int32_t mv = moves[t];
        int kind = mv_kind(mv), qc = mv_qc(mv);
        if (kind == MV_INSERT) {
            out.push_back(Res{-1, (uint8_t)qc, -1});
            continue;
        }
        const Node& pre = g.node[w.row_node[mv_row(mv)]];
        if (kind == MV_MATCH) {
            out.push_back(Res{pre.id, pre.base, -1});
        } else {
            const Node& par = g.node[pre.par_id];
            if (par.aligned[qc] != -1) out.push_back(Res{par.aligned[qc], (uint8_t)qc, -1});
            else out.push_back(Res{-1, (uint8_t)qc, pre.par_id});
        }
    }
}

// graph::output_gfa, src/graph.cpp:358-434. Segments and links come out in
// FIFO Kahn order from the source, which stops at the sink; links follow each
// node's in-list (edges from the source are not written). A read's path is
// its node per position, from the (read ord, position) pairs its nodes carry.
// A read with no bases gets "P\t<name>\t" and no line end, as in the
// reference, which writes the terminator after the last position only.
void Graph::gfa_text(const std::vector<int32_t>& read_len, const std::vector<std::string>& names,
                     const std::vector<int32_t>& rid_to_ord, std::string& out) const {
    out.clear();
    const int n = (int)node.size();
    if (n <= 2) return;
    const int nseq = (int)read_len.size();
    std::vector<int32_t> deg(n);
    for (int i = 0; i < n; i++) deg[i] = (int32_t)node[i].in.size();
    std::vector<std::vector<int32_t>> paths(nseq);
    for (int i = 0; i < nseq; i++) paths[i].assign(read_len[rid_to_ord[i]], 0);
    out += "H\tVN:Z:1.0\n";
    std::vector<int32_t> fifo;
    fifo.reserve(n);
    fifo.push_back(0);
    for (size_t head = 0; head < fifo.size(); head++) {
        const int cur = fifo[head];
        if (cur == 1) break;
        const Node& v = node[cur];
        if (cur != 0) {
            out += "S\t" + std::to_string(cur - 1) + "\t" + kNt256[v.base] + "\n";
            for (int32_t pre : v.in)
                if (pre != 0) out += "L\t" + std::to_string(pre - 1) + "\t+\t" + std::to_string(cur - 1) + "\t+\t0M\n";
            for (size_t k = 0; k < v.ids.size() && k < v.idp.size(); k++) {
                const int id = v.ids[k], pos = v.idp[k];
                if (id >= 0 && id < nseq && pos >= 0 && pos < (int)paths[id].size()) paths[id][pos] = cur - 1;
            }
        }
        for (int32_t o : v.out)
            if (--deg[o] == 0) fifo.push_back(o);
    }
    for (int i = 0; i < nseq; i++) {
        out += "P\t";
        out += (i < (int)names.size() && !names[i].empty()) ? names[i] : std::to_string(i + 1);
        out += "\t";
        const std::vector<int32_t>& pth = paths[rid_to_ord[i]];
        const int len = (int)paths[i].size();
        for (int j = 0; j < len; j++) {
            out += std::to_string(j < (int)pth.size() ? pth[j] : 0);
            out += j + 1 < len ? "+," : "+\t*\n";
        }
    }
}

}  // namespace pb
