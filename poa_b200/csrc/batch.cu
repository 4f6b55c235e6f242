// batch.cu - persistent batched POA over independent windows (see batch.h).
//
// Device graph. A window's graph lives in its warp's slot as flat arrays with
// fixed capacities: per node base, par_id, aligned_node[5], in-degree count,
// rank and the heads/tails of two singly linked edge lists (in-list and
// out-list, kept in insertion order exactly like node_t's vectors); per edge
// its endpoints, weight and the next links of both lists. One warp runs a
// window: fusion (src/graph.cpp:170-235) is warp-parallel with stamp-based
// conflict detection and a sequential fallback (dg_fuse_warp / dg_fuse_seq);
// the LIFO topological sort (src/graph.cpp:21-128) runs its Kahn loop over a
// shared-memory CSR copy, with hlen/tlen as depths by pointer jumping over
// the warp; the window view of the DP rows, the shifted query, the fill and
// the static-band backtrack use the whole warp; the adaptive-band backtrack
// and the consensus (src/graph.cpp:294-351) are the reference's sequential
// walks, run by lane 0.
#include "batch.h"
#include "proposer.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <stdexcept>

#include "gpu_engine.h"
#include "plain.cuh"

namespace pb {

namespace {

inline size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

struct SlotLayout {
    int32_t NC, EC, QC;         // node, edge and query capacities
    int32_t ring_rows, ring_blocks;
    int64_t rs_cap, tb_cap;     // int32 units / bytes
    // byte offsets inside a slot
    int64_t hdr, base, par, aligned, ind, rank, in_head, in_tail, out_head, out_tail, in_cnt, out_cnt;
    int64_t e_from, e_to, e_w, e_nin, e_nout;
    int64_t rank_to_id, hlen, tlen, deg, stk, pre, score, hin, hout, stamp;
    int64_t v_in_ptr, v_in_row, v_in_w, v_in_base, v_out_ptr, v_out_row, v_base, v_ind, v_hq, v_hq_loc, v_tq;
    int64_t v_pmeta, v_desc;
    int64_t meta, state, qs, moves, path, rs, tb;
    int64_t bytes;
};

SlotLayout make_layout(int32_t NC, int32_t EC, int32_t QC, int32_t ring_rows, int32_t ring_blocks, int64_t spill,
                       int64_t tb_cap, bool adaptive) {
    SlotLayout L;
    std::memset(&L, 0, sizeof L);
    L.NC = NC; L.EC = EC; L.QC = QC;
    L.ring_rows = ring_rows; L.ring_blocks = ring_blocks;
    L.rs_cap = (int64_t)ring_rows * ring_blocks * 16 + spill;
    L.tb_cap = tb_cap;
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t r = o; o = up256(o + bytes); return (int64_t)r; };
    const size_t n4 = 4 * (size_t)NC, e4 = 4 * (size_t)EC;
    L.hdr = take(64);
    L.base = take(NC); L.par = take(n4); L.aligned = take(5 * n4); L.ind = take(n4); L.rank = take(n4);
    L.in_head = take(n4); L.in_tail = take(n4); L.out_head = take(n4); L.out_tail = take(n4);
    L.in_cnt = take(n4); L.out_cnt = take(n4);
    L.e_from = take(e4); L.e_to = take(e4); L.e_w = take(e4); L.e_nin = take(e4); L.e_nout = take(e4);
    L.rank_to_id = take(n4); L.hlen = take(n4); L.tlen = take(n4); L.deg = take(n4); L.stk = take(n4);
    L.pre = take(n4); L.score = take(n4);
    L.hin = take(n4); L.hout = take(n4); L.stamp = take(n4);
    L.v_in_ptr = take(n4 + 4); L.v_in_row = take(e4); L.v_in_w = take(e4); L.v_in_base = take(EC);
    L.v_out_ptr = take(n4 + 4); L.v_out_row = take(e4); L.v_base = take(NC); L.v_ind = take(n4);
    L.v_hq = take(n4); L.v_hq_loc = take(n4); L.v_tq = take(n4);
    L.v_pmeta = take(16 * (size_t)EC);
    L.v_desc = take(48 * (size_t)NC);
    L.meta = take(sizeof(RowMeta) * (size_t)NC);
    L.state = take(adaptive ? 4 * (size_t)AB_NSTATE * NC : 64);
    L.qs = take((size_t)qs_bytes(QC) + 64);
    L.moves = take(4 * ((size_t)NC + QC + 16));
    L.path = take(4 * ((size_t)NC + QC + 16));
    L.rs = take(4 * (size_t)L.rs_cap);
    L.tb = take((size_t)tb_cap);
    L.bytes = (int64_t)up256(o);
    return L;
}

struct BatchArgs {
    const uint8_t* seq;
    const int64_t* read_off;
    const int32_t* read_len;
    const int32_t* win_off;
    const int32_t* order;
    int32_t* counter;
    int32_t n_windows;
    Scoring sc;
    int32_t b, f, ab_band;
    char* slots;
    SlotLayout L;
    int32_t smem_per_warp;   // bytes of dynamic shared memory per warp
    int32_t sring_rows;      // shared-memory ring rows of the static-band fill (0 = all rows in global)
    int32_t sring_blocks;    // blocks per ring row
    char* cons;
    int32_t cons_stride;
    int32_t* cons_len;
    int32_t* status;
    int64_t* cells;  // [n_windows * 2] band cells and edge-cells (cells x in-window predecessors)
    int64_t* phase;  // [n_windows * NPHASE] lane-0 clock cycles per phase
    int32_t* rstats; // [n_reads * NRSTAT] per read, see BatchEngine::read_stats
};

// per-window cycle counters (clock64 on lane 0): where a window's time goes
enum { PH_VIEW = 0, PH_FILL, PH_BT, PH_FUSE, PH_SORT, PH_CONS, NPHASE = 8 };

// Pointers of one slot's device graph.
struct DevGraph {
    int32_t* hdr;  // [0] nodes, [1] edges, [2] status, [3] ranks, [4..11] DP outputs, [12] fusion stamp, [13] moves
    uint8_t* base;
    int32_t *par, *aligned, *ind, *rank, *in_head, *in_tail, *out_head, *out_tail, *in_cnt, *out_cnt;
    int32_t *e_from, *e_to, *e_w, *e_nin, *e_nout;
    int32_t *rank_to_id, *hlen, *tlen, *deg, *stk, *pre, *score;
    int32_t *hin, *hout, *stamp;  // heaviest in/out edge (first max in list order); fusion stamps
    int32_t *csr_ptr, *csr_adj;   // topsort scratch: the view's out-lists, free until the view is rebuilt
    int32_t NC, EC;
};

__device__ DevGraph slot_graph(char* s, const SlotLayout& L) {
    DevGraph g;
    g.hdr = (int32_t*)(s + L.hdr);
    g.base = (uint8_t*)(s + L.base);
    g.par = (int32_t*)(s + L.par); g.aligned = (int32_t*)(s + L.aligned); g.ind = (int32_t*)(s + L.ind);
    g.rank = (int32_t*)(s + L.rank);
    g.in_head = (int32_t*)(s + L.in_head); g.in_tail = (int32_t*)(s + L.in_tail);
    g.out_head = (int32_t*)(s + L.out_head); g.out_tail = (int32_t*)(s + L.out_tail);
    g.in_cnt = (int32_t*)(s + L.in_cnt); g.out_cnt = (int32_t*)(s + L.out_cnt);
    g.e_from = (int32_t*)(s + L.e_from); g.e_to = (int32_t*)(s + L.e_to); g.e_w = (int32_t*)(s + L.e_w);
    g.e_nin = (int32_t*)(s + L.e_nin); g.e_nout = (int32_t*)(s + L.e_nout);
    g.rank_to_id = (int32_t*)(s + L.rank_to_id); g.hlen = (int32_t*)(s + L.hlen); g.tlen = (int32_t*)(s + L.tlen);
    g.deg = (int32_t*)(s + L.deg); g.stk = (int32_t*)(s + L.stk); g.pre = (int32_t*)(s + L.pre);
    g.score = (int32_t*)(s + L.score);
    g.hin = (int32_t*)(s + L.hin); g.hout = (int32_t*)(s + L.hout); g.stamp = (int32_t*)(s + L.stamp);
    g.csr_ptr = (int32_t*)(s + L.v_out_ptr); g.csr_adj = (int32_t*)(s + L.v_out_row);
    g.NC = L.NC; g.EC = L.EC;
    return g;
}

__device__ __forceinline__ uint8_t nt4_dev(uint8_t c) {
    switch (c) {
        case 0: case 1: case 2: case 3: return c;
        case 'A': case 'a': return 0;
        case 'C': case 'c': return 1;
        case 'G': case 'g': return 2;
        case 'T': case 't': case 'U': case 'u': return 3;
        default: return 4;
    }
}

// node_t ctor (include/node.h:16-22); -1 when the slot is full
__device__ int dg_add_node(DevGraph& g, int& nn, uint8_t base) {
    if (nn >= g.NC) return -1;
    const int id = nn++;
    g.base[id] = base;
    g.par[id] = id;
#pragma unroll
    for (int k = 0; k < 5; k++) g.aligned[id * 5 + k] = -1;
    g.aligned[id * 5 + base] = id;
    g.ind[id] = 0;
    g.in_head[id] = g.in_tail[id] = g.out_head[id] = g.out_tail[id] = -1;
    g.in_cnt[id] = g.out_cnt[id] = 0;
    g.hin[id] = g.hout[id] = -1;
    g.stamp[id] = 0;
    return id;
}

// Keep hin[v] / hout[u] = the heaviest in/out edge, first in list order on
// ties, after edge e (u -> v) gained weight or was appended. List order is
// edge-id order (edges are only ever appended), and only e changed, so the new
// heaviest is the old one or e.
__device__ __forceinline__ void dg_heavy(DevGraph& g, int e, int u, int v) {
    const int w = g.e_w[e];
    int b = g.hin[v];
    if (b < 0 || w > g.e_w[b] || (w == g.e_w[b] && e < b)) g.hin[v] = e;
    b = g.hout[u];
    if (b < 0 || w > g.e_w[b] || (w == g.e_w[b] && e < b)) g.hout[u] = e;
}

// graph::add_adj (src/graph.cpp:13-20, include/node.h:23-61); false when full
__device__ bool dg_add_adj(DevGraph& g, int& ne, int u, int v) {
    if (u == v) return true;
    g.ind[v]++;
    for (int e = g.out_head[u]; e >= 0; e = g.e_nout[e])
        if (g.e_to[e] == v) {
            g.e_w[e]++;
            dg_heavy(g, e, u, v);
            return true;
        }
    if (ne >= g.EC) return false;
    const int e = ne++;
    g.e_from[e] = u; g.e_to[e] = v; g.e_w[e] = 1; g.e_nin[e] = -1; g.e_nout[e] = -1;
    if (g.out_tail[u] >= 0) g.e_nout[g.out_tail[u]] = e; else g.out_head[u] = e;
    g.out_tail[u] = e; g.out_cnt[u]++;
    if (g.in_tail[v] >= 0) g.e_nin[g.in_tail[v]] = e; else g.in_head[v] = e;
    g.in_tail[v] = e; g.in_cnt[v]++;
    dg_heavy(g, e, u, v);
    return true;
}

// graph::topsort op 0 (src/graph.cpp:61-123), lane 0 only; returns #ranks
__device__ int dg_topsort(DevGraph& g, int nn, bool with_lens) {
    int sp = 0, nr = 0;
    for (int i = 0; i < nn; i++) {
        g.deg[i] = g.in_cnt[i];
        if (g.deg[i] == 0) g.stk[sp++] = i;
    }
    while (sp) {
        const int u = g.stk[--sp];
        g.rank[u] = nr;
        g.rank_to_id[nr++] = u;
        for (int e = g.out_head[u]; e >= 0; e = g.e_nout[e]) {
            const int v = g.e_to[e];
            if (--g.deg[v] == 0) g.stk[sp++] = v;
        }
    }
    if (with_lens) {
        for (int i = 0; i < nr; i++) {
            const int u = g.rank_to_id[i];
            int wmax = -1, max_pre = -1;
            for (int e = g.in_head[u]; e >= 0; e = g.e_nin[e])
                if (g.e_w[e] > wmax) { wmax = g.e_w[e]; max_pre = g.rank[g.e_from[e]]; }
            if (max_pre != -1) g.hlen[g.rank[u]] = g.hlen[max_pre] + 1;
        }
        g.tlen[g.rank[1]] = 1;
        for (int i = nr - 1; i >= 0; i--) {
            const int u = g.rank_to_id[i];
            int wmax = -1, max_suc = -1;
            for (int e = g.out_head[u]; e >= 0; e = g.e_nout[e])
                if (g.e_w[e] > wmax) { wmax = g.e_w[e]; max_suc = g.rank[g.e_to[e]]; }
            if (max_suc != -1) g.tlen[g.rank[u]] = g.tlen[max_suc] + 1;
        }
    }
    return nr;
}

// graph::build_consensus (src/graph.cpp:294-351), lane 0; returns its length
// (or -1 when it does not fit into cap) and writes ASCII to out
__device__ int dg_consensus(DevGraph& g, int nn, char* out, int cap) {
    int qh = 0, qt = 0;
    for (int i = 0; i < nn; i++) { g.deg[i] = g.in_cnt[i]; g.pre[i] = 0; g.score[i] = 0; }
    g.stk[qt++] = 0;
    while (qh < qt) {
        const int u = g.stk[qh++];
        if (u != 0) {
            int wmax = -1, max_pre = -1;
            for (int e = g.in_head[u]; e >= 0; e = g.e_nin[e]) {
                const int pr = g.e_from[e], wk = g.e_w[e];
                if (wk > wmax || (wk == wmax && g.score[pr] > g.score[max_pre])) { wmax = wk; max_pre = pr; }
            }
            g.pre[u] = max_pre;
            g.score[u] = g.score[max_pre] + wmax;
        }
        if (u == 1) break;
        for (int e = g.out_head[u]; e >= 0; e = g.e_nout[e])
            if (--g.deg[g.e_to[e]] == 0) g.stk[qt++] = g.e_to[e];
    }
    int len = 0;
    for (int id = g.pre[1]; id != 0; id = g.pre[id]) len++;
    if (len > cap) return -1;
    const char nt[5] = {'A', 'C', 'G', 'T', 'N'};
    int k = len;
    for (int id = g.pre[1]; id != 0; id = g.pre[id]) out[--k] = nt[g.base[id]];
    return len;
}

// Sequential fusion of one backtrack path (lane 0): the reference's order of
// node creation and edge insertion, one element at a time.
__device__ int dg_fuse_seq(DevGraph& g, const int32_t* moves, int nm, int beg_i) {
    int st = ST_OK;
    int nn = g.hdr[0], ne = g.hdr[1], anchored = -1;
    for (int t = nm - 1; t >= 0 && st == ST_OK; t--) {
        const int32_t mv = moves[t];
        const int kind = mv_kind(mv), qc = mv_qc(mv);
        int cur;
        if (kind == MV_INSERT) {
            cur = dg_add_node(g, nn, (uint8_t)qc);
        } else {
            const int pre = g.rank_to_id[beg_i + mv_row(mv)];
            if (kind == MV_MATCH) {
                cur = pre;
            } else {
                const int par = g.par[pre];
                cur = g.aligned[par * 5 + qc];
                if (cur == -1) {
                    cur = dg_add_node(g, nn, (uint8_t)qc);
                    if (cur >= 0) {
                        g.aligned[par * 5 + qc] = cur;
                        g.par[cur] = par;
                    }
                }
            }
        }
        if (cur < 0) { st = ST_CAPACITY; break; }
        if (anchored != -1 && !dg_add_adj(g, ne, anchored, cur)) st = ST_CAPACITY;
        anchored = cur;
    }
    if (st == ST_OK && !dg_add_adj(g, ne, anchored, 1)) st = ST_CAPACITY;
    g.hdr[0] = nn;
    g.hdr[1] = ne;
    return st;
}

// Fusion of one backtrack path with the whole warp (src/graph.cpp:170-235,
// path elements as emitted by src/align.cpp:1606-1620, 1672-1682).
// Path element q (backtrack move nm-1-q) becomes a node id: the predecessor
// row's node for a match, its parent's aligned sibling for a mismatch (new
// when absent), a new node for an insertion. New nodes get ids in path order
// (prefix sums). The path then adds edges (q -> q+1) and (last -> sink); in a
// path every node occurs once, so every in-list, out-list, in-degree and
// heaviest-edge slot is touched by one edge at most and the edges are applied
// in parallel. A path that would create the same aligned node twice or visit
// a node twice is detected (CAS claims, fusion stamps) and fused sequentially
// instead. Returns ST_OK, ST_CAPACITY, or -1 for "use the sequential path".
__device__ int dg_fuse_warp(DevGraph& g, const int32_t* moves, int nm, int beg_i, int32_t* path, int fid,
                            int lane) {
    const int nn0 = g.hdr[0], ne0 = g.hdr[1];
    const unsigned lt = (1u << lane) - 1u;
    bool conflict = false, full = false;
    int new_total = 0;
    for (int c0 = 0; c0 < nm; c0 += 32) {
        const int q = c0 + lane;
        bool is_new = false;
        int cur = -1, par = -1, qc = 0, kind = MV_INSERT;
        if (q < nm) {
            const int32_t mv = moves[nm - 1 - q];
            kind = mv_kind(mv);
            qc = mv_qc(mv);
            if (kind == MV_INSERT) {
                is_new = true;
            } else {
                const int pre = g.rank_to_id[beg_i + mv_row(mv)];
                if (kind == MV_MATCH) {
                    cur = pre;
                } else {
                    par = g.par[pre];
                    cur = g.aligned[par * 5 + qc];
                    is_new = cur == -1;
                }
            }
        }
        const unsigned msk = __ballot_sync(0xffffffffu, is_new);
        if (is_new) {
            cur = nn0 + new_total + __popc(msk & lt);
            if (cur >= g.NC) {
                full = true;
            } else {
                g.base[cur] = (uint8_t)qc;
                g.par[cur] = par >= 0 ? par : cur;
#pragma unroll
                for (int k = 0; k < 5; k++) g.aligned[cur * 5 + k] = -1;
                g.aligned[cur * 5 + qc] = cur;
                g.ind[cur] = 0;
                g.in_head[cur] = g.in_tail[cur] = g.out_head[cur] = g.out_tail[cur] = -1;
                g.in_cnt[cur] = g.out_cnt[cur] = 0;
                g.hin[cur] = g.hout[cur] = -1;
                if (par >= 0 && atomicCAS(&g.aligned[par * 5 + qc], -1, cur) != -1) conflict = true;
            }
        }
        if (q < nm && cur >= 0 && cur < g.NC && atomicExch(&g.stamp[cur], fid) == fid) conflict = true;
        if (q < nm) path[q] = cur;
        new_total += __popc(msk);
    }
    const bool any_full = __any_sync(0xffffffffu, full);
    const bool any_conflict = __any_sync(0xffffffffu, conflict);
    if (any_full || any_conflict) {
        // undo this path's aligned claims; the node slots past nn0 are simply not kept
        __syncwarp();
        for (int q = lane; q < nm; q += 32) {
            const int cur = path[q];
            if (cur >= nn0 && cur < g.NC && g.par[cur] != cur) {
                const int par = g.par[cur];
                atomicCAS(&g.aligned[par * 5 + g.base[cur]], cur, -1);
            }
        }
        __syncwarp();
        return any_full ? ST_CAPACITY : -1;
    }
    __syncwarp();
    // edges: pair t joins path[t] -> path[t+1] (the last one -> sink)
    int new_edges = 0;
    bool efull = false;
    for (int c0 = 0; c0 < nm; c0 += 32) {
        const int t = c0 + lane;
        int u = -1, v = -1, found = -1;
        bool need = false;
        if (t < nm) {
            u = path[t];
            v = t + 1 < nm ? path[t + 1] : 1;
            if (u != v) {
                for (int e = g.out_head[u]; e >= 0; e = g.e_nout[e])
                    if (g.e_to[e] == v) { found = e; break; }
                need = found < 0;
            }
        }
        const unsigned msk = __ballot_sync(0xffffffffu, need);
        if (t < nm && u != v) {
            g.ind[v]++;
            if (found >= 0) {
                g.e_w[found]++;
                dg_heavy(g, found, u, v);
            } else {
                const int e = ne0 + new_edges + __popc(msk & lt);
                if (e >= g.EC) {
                    efull = true;
                } else {
                    g.e_from[e] = u; g.e_to[e] = v; g.e_w[e] = 1; g.e_nin[e] = -1; g.e_nout[e] = -1;
                    if (g.out_tail[u] >= 0) g.e_nout[g.out_tail[u]] = e; else g.out_head[u] = e;
                    g.out_tail[u] = e; g.out_cnt[u]++;
                    if (g.in_tail[v] >= 0) g.e_nin[g.in_tail[v]] = e; else g.in_head[v] = e;
                    g.in_tail[v] = e; g.in_cnt[v]++;
                    dg_heavy(g, e, u, v);
                }
            }
        }
        new_edges += __popc(msk);
        __syncwarp();
    }
    if (__any_sync(0xffffffffu, efull)) return ST_CAPACITY;
    if (lane == 0) {
        g.hdr[0] = nn0 + new_total;
        g.hdr[1] = ne0 + new_edges;
    }
    __syncwarp();
    return ST_OK;
}

// Depth of every node in the forest where each node's parent is the far end
// of its heaviest in-edge (pass 0, hlen: src/graph.cpp:86-101) or heaviest
// out-edge (pass 1, tlen: src/graph.cpp:103-121). Roots keep the value the
// array already holds at their rank (the reference resizes the vector and
// never writes there), except the sink, whose tlen is 1. Written back by rank.
template <typename T>
__device__ void depth_jump(DevGraph& g, int nn, int pass, int32_t* arr, T* P, T* Q, T* D, T* E, int lane) {
    const T none = (T)-1;
    for (int u = lane; u < nn; u += 32) {
        const int e = pass == 0 ? g.hin[u] : g.hout[u];
        const int par = e < 0 ? -1 : (pass == 0 ? g.e_from[e] : g.e_to[e]);
        P[u] = par < 0 ? none : (T)par;
        D[u] = par >= 0 ? (T)1 : (T)((pass == 1 && u == 1) ? 1 : arr[g.rank[u]]);
    }
    __syncwarp();
    for (int it = 0; it < 40; it++) {
        bool moved = false;
        for (int u = lane; u < nn; u += 32) {
            const T p = P[u];
            if (p != none) {
                E[u] = (T)(D[u] + D[p]);
                Q[u] = P[p];
                moved = true;
            } else {
                E[u] = D[u];
                Q[u] = none;
            }
        }
        __syncwarp();
        T* t = P; P = Q; Q = t;
        t = D; D = E; E = t;
        if (!__any_sync(0xffffffffu, moved)) break;
    }
    for (int u = lane; u < nn; u += 32) arr[g.rank[u]] = (int32_t)D[u];
    __syncwarp();
}

// Topological sort with the whole warp: the out-lists are copied into
// shared memory as CSR (16-bit ids), the LIFO Kahn loop of
// src/graph.cpp:61-85 then runs on lane 0 over shared memory only, and
// hlen/tlen (src/graph.cpp:86-123) are depths in the heaviest-in-edge and
// heaviest-out-edge forests, computed by pointer jumping across the warp
// (double-buffered in the slot's scratch arrays). Graphs too large for the
// shared-memory budget use the sequential global-memory version.
// The same LIFO Kahn order for graphs whose 16-bit lists do not fit the warp's
// shared memory: out-lists as int32 CSR in the slot's view arrays, in-degree
// counters (8 bits) and the stack (16 bits) in shared memory. Returns false
// when an in-degree exceeds 255 or the stack outgrows its space; the caller
// then sorts on the global lists, which recomputes every rank.
__device__ bool topsort_large(DevGraph& g, int nn, uint8_t* sm, int sm_bytes, int lane) {
    int32_t* optr = g.csr_ptr;
    int32_t* adj = g.csr_adj;
    uint8_t* deg = sm;
    uint16_t* stk = reinterpret_cast<uint16_t*>(sm + ((nn + 15) & ~15));
    const int cap = (sm_bytes - ((nn + 15) & ~15)) / 2;
    int carry = 0;
    bool big = false;
    for (int c0 = 0; c0 < nn; c0 += 32) {
        const int u = c0 + lane;
        const int c = u < nn ? g.out_cnt[u] : 0;
        int x = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (u < nn) optr[u] = carry + x - c;
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0) optr[nn] = carry;
    for (int u = lane; u < nn; u += 32) {
        int k = optr[u];
        for (int e = g.out_head[u]; e >= 0; e = g.e_nout[e]) adj[k++] = g.e_to[e];
        const int ic = g.in_cnt[u];
        big |= ic > 255;
        deg[u] = (uint8_t)ic;
    }
    if (__any_sync(0xffffffffu, big)) return false;
    // zero in-degree seeds in id order
    int sp = 0;
    bool over = false;
    for (int c0 = 0; c0 < nn; c0 += 32) {
        const int u = c0 + lane;
        const bool z = u < nn && deg[u] == 0;
        const unsigned msk = __ballot_sync(0xffffffffu, z);
        over |= sp + __popc(msk) > cap;
        if (z && !over) stk[sp + __popc(msk & ((1u << lane) - 1u))] = (uint16_t)u;
        sp += __popc(msk);
    }
    __syncwarp();
    if (over) return false;
    int nr = 0;
    if (lane == 0) {
        while (sp && !over) {
            const int u = stk[--sp];
            g.rank[u] = nr;
            g.rank_to_id[nr++] = u;
            const int k1 = optr[u + 1];
            for (int k = optr[u]; k < k1; k++) {
                const int v = adj[k];
                const int dv = deg[v] - 1;
                deg[v] = (uint8_t)dv;
                if (dv == 0) {
                    if (sp >= cap) { over = true; break; }
                    stk[sp++] = (uint16_t)v;
                }
            }
        }
        if (!over) g.hdr[3] = nr;
    }
    over = __shfl_sync(0xffffffffu, over, 0);
    __syncwarp();
    return !over;
}

__device__ void dg_topsort_warp(DevGraph& g, int nn, int ne, bool with_lens, uint16_t* sm, int sm_bytes,
                                int lane) {
    const size_t need = 2 * ((size_t)nn + 1) + 2 * (size_t)ne + 4 * (size_t)nn + 16;
    if (nn >= 65535 || ne >= 65535 || need > (size_t)sm_bytes) {
        if (nn < 65535 && (size_t)nn + 16 + 2 * 256 <= (size_t)sm_bytes) {
            if (topsort_large(g, nn, (uint8_t*)sm, sm_bytes, lane)) {
                if (with_lens)
                    for (int pass = 0; pass < 2; pass++)
                        depth_jump<int32_t>(g, nn, pass, pass == 0 ? g.hlen : g.tlen, g.deg, g.stk, g.pre, g.score,
                                            lane);
                return;
            }
        }
        if (lane == 0) g.hdr[3] = dg_topsort(g, nn, with_lens);
        __syncwarp();
        return;
    }
    uint16_t* optr = sm;
    uint16_t* adj = optr + nn + 1;
    uint16_t* deg = adj + ne;
    uint16_t* stk = deg + nn;
    int carry = 0;
    for (int c0 = 0; c0 < nn; c0 += 32) {
        const int u = c0 + lane;
        const int c = u < nn ? g.out_cnt[u] : 0;
        int x = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (u < nn) optr[u] = (uint16_t)(carry + x - c);
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0) optr[nn] = (uint16_t)carry;
    for (int u = lane; u < nn; u += 32) {
        int k = 0;
        const int base_k = (int)optr[u];
        for (int e = g.out_head[u]; e >= 0; e = g.e_nout[e]) adj[base_k + k++] = (uint16_t)g.e_to[e];
        deg[u] = (uint16_t)g.in_cnt[u];
    }
    __syncwarp();
    // zero in-degree seeds in id order
    int sp = 0;
    for (int c0 = 0; c0 < nn; c0 += 32) {
        const int u = c0 + lane;
        const bool z = u < nn && deg[u] == 0;
        const unsigned msk = __ballot_sync(0xffffffffu, z);
        if (z) stk[sp + __popc(msk & ((1u << lane) - 1u))] = (uint16_t)u;
        sp += __popc(msk);
    }
    __syncwarp();
    if (lane == 0) {
        int nr = 0;
        while (sp) {
            const int u = stk[--sp];
            g.rank[u] = nr;
            g.rank_to_id[nr++] = u;
            const int k1 = optr[u + 1];
            for (int k = optr[u]; k < k1; k++) {
                const int v = adj[k];
                const int dv = deg[v] - 1;
                deg[v] = (uint16_t)dv;
                if (dv == 0) stk[sp++] = (uint16_t)v;
            }
        }
        g.hdr[3] = nr;
    }
    __syncwarp();
    if (!with_lens) return;
    // hlen / tlen: depths in the forests of heaviest in-edges (hin) and
    // heaviest out-edges (hout), by pointer jumping; 16-bit arrays in shared
    // memory when they fit, the slot's int32 scratch otherwise
    const bool sm_ok = 8 * (size_t)nn + 16 <= (size_t)sm_bytes;
    for (int pass = 0; pass < 2; pass++) {
        int32_t* arr = pass == 0 ? g.hlen : g.tlen;
        if (sm_ok) depth_jump<uint16_t>(g, nn, pass, arr, sm, sm + nn, sm + 2 * nn, sm + 3 * nn, lane);
        else depth_jump<int32_t>(g, nn, pass, arr, g.deg, g.stk, g.pre, g.score, lane);
    }
}

// Everything the static-band fill needs about one row, in one 48-byte record
// (three 16-byte loads, issued one row ahead): the band, where the row's M/D
// blocks and records go, its predecessor range, and the first predecessor's
// band/location/base/weight so single-predecessor rows need nothing else.
struct __align__(16) RowDesc {
    int32_t bsbe, st, tb, e0;      // Bs | Be << 16, row store location, record offset, first in-edge
    int32_t d, ind, w1ok, prow0;   // in-window predecessors, in-degree count, in_weight >= ind/10, first pred row
    int32_t pbsbe, pst, pbase, pw; // first predecessor: band, location, base (as the DP sees it), in_weight
};

// Static-band view (f > 0, no adaptive band): besides the predecessor lists,
// every row's band, row-store location and record offset are a pure function
// of hlen/tlen, so the warp computes them all here, in parallel, and attaches
// to each in-edge the predecessor's (Bs, Be, location). The fill then needs
// one coalesced load per predecessor and no per-row bookkeeping.
// Row store location: ring slot -(r % R) - 1 in shared memory, or an offset
// in the slot's spill area for rows with a successor R or more rows ahead.
__device__ int build_view_static(DevGraph& g, char* s, const SlotLayout& L, WinView& v, int m, int f, int wband,
                                 int R, int RB, int lane, int& beg_out) {
    const int beg_i = g.rank[0], end_i = g.rank[1];
    const int n = end_i - beg_i + 1;
    beg_out = beg_i;
    int32_t* in_ptr = (int32_t*)(s + L.v_in_ptr);
    int32_t* in_row = (int32_t*)(s + L.v_in_row);
    int32_t* in_w = (int32_t*)(s + L.v_in_w);
    uint8_t* in_base = (uint8_t*)(s + L.v_in_base);
    int32_t* vind = (int32_t*)(s + L.v_ind);
    int4* erec = (int4*)(s + L.v_pmeta);
    RowDesc* desc = (RowDesc*)(s + L.v_desc);
    RowMeta* meta = (RowMeta*)(s + L.meta);
    const int h0 = g.hlen[beg_i], t0 = g.tlen[end_i];
    const int64_t spill_cap = L.rs_cap;
    // pass 1: per-row counts, band, widths
    for (int r = lane; r < n; r += 32) {
        const int u = g.rank_to_id[beg_i + r];
        int ci = 0, maxs = r;
        for (int e = g.in_head[u]; e >= 0; e = g.e_nin[e]) ci += (g.rank[g.e_from[e]] - beg_i >= 0);
        for (int e = g.out_head[u]; e >= 0; e = g.e_nout[e]) {
            const int sr = g.rank[g.e_to[e]] - beg_i;
            if (sr < n && sr > maxs) maxs = sr;
        }
        int Bs, Be;
        band_static(f, g.hlen[beg_i + r] - h0, g.tlen[beg_i + r] - t0, m, wband, Bs, Be);
        if (r == 0) Bs = 0;
        const int bn = Be - Bs - 1;
        const int d = r == 0 ? 0 : ci;
        const int bpc = d >= 2 ? 4 : 1;
        const bool spill = R == 0 || (maxs - r >= R) || bn > RB;
        in_ptr[r + 1] = ci;
        vind[r] = g.ind[u];
        RowMeta rm;
        rm.Bs = Bs;
        rm.Be = Be;
        rm.tb = bn > 0 ? (((int64_t)bn * BLK * bpc + 15) & ~(int64_t)15) : 0;   // widths, scanned below
        rm.st = spill ? (bn > 0 ? (int64_t)bn * 16 : 0) : -1;
        if (bn < 0 || d > MAX_MULTI_PRED) rm.Be = INT32_MIN;                  // flagged
        meta[r] = rm;
    }
    __syncwarp();
    // scans: in_ptr, record offsets, spill offsets
    int ci_c = 0;
    int64_t tb_c = 0, sp_c = 0;
    bool bad = false;
    if (lane == 0) in_ptr[0] = 0;
    for (int c0 = 0; c0 < n; c0 += 32) {
        const int r = c0 + lane;
        RowMeta rm;
        int ci = 0;
        int64_t tbw = 0, spw = 0;
        bool sp = false;
        if (r < n) {
            rm = meta[r];
            ci = in_ptr[r + 1];
            tbw = rm.tb;
            sp = rm.st >= 0;
            spw = sp ? rm.st : 0;
            bad |= rm.Be == INT32_MIN;
        }
        int xi = ci;
        long long xt = tbw, xs = spw;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int yi = __shfl_up_sync(0xffffffffu, xi, o);
            const long long yt = __shfl_up_sync(0xffffffffu, xt, o);
            const long long ys = __shfl_up_sync(0xffffffffu, xs, o);
            if (lane >= o) { xi += yi; xt += yt; xs += ys; }
        }
        if (r < n) {
            in_ptr[r + 1] = ci_c + xi;
            rm.tb = tb_c + (xt - tbw);
            rm.st = sp ? sp_c + (xs - spw) : -(int64_t)(r % (R > 0 ? R : 1)) - 1;
            meta[r] = rm;
        }
        ci_c += __shfl_sync(0xffffffffu, xi, 31);
        tb_c += __shfl_sync(0xffffffffu, xt, 31);
        sp_c += __shfl_sync(0xffffffffu, xs, 31);
    }
    if (lane == 0) {
        g.hdr[8] = (int32_t)(tb_c > INT_MAX ? INT_MAX : tb_c);   // DP output 4: record bytes
        g.hdr[9] = (int32_t)(sp_c > INT_MAX ? INT_MAX : sp_c);   // DP output 5: spilled row-store entries
    }
    if (__any_sync(0xffffffffu, bad)) return ST_DEGENERATE;
    if (tb_c > L.tb_cap || sp_c > spill_cap) return ST_OOM;
    __syncwarp();
    // pass 2: predecessor lists in in-list order
    for (int r = lane; r < n; r += 32) {
        const int u = g.rank_to_id[beg_i + r];
        int k = in_ptr[r];
        for (int e = g.in_head[u]; e >= 0; e = g.e_nin[e]) {
            const int p = g.rank[g.e_from[e]] - beg_i;
            if (p < 0) continue;
            in_row[k] = p;
            in_w[k] = g.e_w[e];
            in_base[k] = p == 0 ? 4 : g.base[g.e_from[e]];
            k++;
        }
    }
    __syncwarp();
    // pass 3: each row's predecessor records in the backtrack's priority order
    // (in_weight descending, in-list position ascending; src/align.cpp:1601,
    // 1637, 1708 keep the first maximum), so the fill can take "the first
    // predecessor that satisfies a test" as the backtrack's choice.
    // erec = {Bs | Be << 16, row-store location, in_weight | position << 16,
    //         base | (in_weight >= ind/10) << 8}
    for (int r = lane; r < n; r += 32) {
        const int e0 = in_ptr[r], d = r == 0 ? 0 : in_ptr[r + 1] - e0;
        const int ind = vind[r];
        for (int k = 0; k < d; k++) {
            const RowMeta pm = meta[in_row[e0 + k]];
            const int w = in_w[e0 + k];
            const int4 rec = make_int4(pm.Bs | (pm.Be << 16), (int32_t)pm.st, (w & 0xffff) | (k << 16),
                                       (int)in_base[e0 + k] | ((w >= ind / 10) ? 256 : 0));
            // insertion into the sorted prefix [e0, e0 + k)
            int at = k;
            while (at > 0) {
                const int4 prev = erec[e0 + at - 1];
                const int pw = prev.z & 0xffff;
                if (pw >= w) break;  // strictly larger weight moves ahead; ties keep list order
                erec[e0 + at] = prev;
                at--;
            }
            erec[e0 + at] = rec;
        }
    }
    __syncwarp();
    // pass 4: row descriptors (the first predecessor record is the top-priority one)
    for (int r = lane; r < n; r += 32) {
        const RowMeta rm = meta[r];
        const int e0 = in_ptr[r];
        const int d = r == 0 ? 0 : in_ptr[r + 1] - e0;
        RowDesc rd;
        rd.bsbe = rm.Bs | (rm.Be << 16);
        rd.st = (int32_t)rm.st;
        rd.tb = (int32_t)rm.tb;
        rd.e0 = e0;
        rd.d = d;
        rd.ind = vind[r];
        rd.prow0 = d >= 1 ? in_row[e0] : 0;
        if (d >= 1) {
            const int4 er = erec[e0];
            rd.pbsbe = er.x; rd.pst = er.y; rd.pw = er.z & 0xffff; rd.pbase = er.w & 255;
            rd.w1ok = (er.w >> 8) & 1;
        } else {
            rd.pbsbe = rd.pst = rd.pw = rd.pbase = 0;
            rd.w1ok = 0;
        }
        desc[r] = rd;
    }
    __syncwarp();
    v.n = n;
    v.in_ptr = in_ptr; v.in_row = in_row; v.in_w = in_w; v.in_base = in_base;
    v.ind = vind;
    return ST_OK;
}

// Static-band DP fill of one alignment by one warp (see build_view_static).
// Same recurrences and records as dp_fill (plain.cuh), specialised for the
// batch:
//  * row descriptors and predecessor records are staged into shared memory
//    16 rows at a time (one coalesced round trip), so the row loop reads only
//    shared memory: descriptors, predecessor blocks from the shared-memory
//    ring of recent rows (global spill area for rows with distant
//    successors), the query;
//  * the horizontal gap recurrence in the form
//    I[j] = o1 + (j-1)*e1 + max(K, max_{k<j} H0[k]-k*e1), K = NEG_INF+e1-o1,
//    which also yields I[0] = NEG_INF;
//  * records: predecessors arrive in the backtrack's priority order, so each
//    choice (M1 with its weight threshold, M4, D open / extend) is the first
//    predecessor passing its test; single-predecessor rows keep their blocks
//    in registers between the two passes.
constexpr int STAGE_ROWS = 16, STAGE_EDGES = 64;

__device__ __forceinline__ RowDesc load_desc(const RowDesc* p) {
    const int4* q = reinterpret_cast<const int4*>(p);
    const int4 a = q[0], b = q[1], c = q[2];
    RowDesc r;
    r.bsbe = a.x; r.st = a.y; r.tb = a.z; r.e0 = a.w;
    r.d = b.x; r.ind = b.y; r.w1ok = b.z; r.prow0 = b.w;
    r.pbsbe = c.x; r.pst = c.y; r.pbase = c.z; r.pw = c.w;
    return r;
}

__device__ __forceinline__ const int32_t* blk_src(const int32_t* ring, const int32_t* rs, int RB, int st) {
    return st < 0 ? ring + (-st - 1) * RB * 16 : rs + st;
}

// One row of the warp fill: every chunk of 32 blocks (one block per lane) of
// row i, whose descriptor is `cur` and whose predecessor records are
// er_base[cur.e0 + k] in the backtrack's priority order. Predecessor blocks
// come from blk_src (the shared-memory ring or the slot's row store). With
// ARGMAX, each lane also keeps the first maximum of M over its cells.
template <bool ARGMAX, bool TRACK>
__device__ __forceinline__ void fill_row(const DpArgs& a, const RowDesc& cur, const int4* __restrict__ er_base,
                                         const int32_t* ring, int RB, const uint8_t* __restrict__ qsm, int i,
                                         int lane, int32_t& bestM, int& bestJ) {
    const Scoring sc = a.sc;
    const int32_t K = add32(add32(NEG_INF, sc.e1), -sc.o1);
    const int Bs = cur.bsbe & 0xffff, Be = cur.bsbe >> 16, bn = Be - Bs - 1;
    const int d = cur.d;
    int32_t* dst = const_cast<int32_t*>(blk_src(ring, a.rs, RB, cur.st));
    const int nch = (bn + 31) >> 5;
    int32_t carryP = K, carryM = NEG_INF, carryI = NEG_INF;
    for (int c = 0; c < nch; c++) {
        const int b = c * 32 + lane;
        const bool act = b < bn;
        const int B = Bs + b;
        const int j0 = b * BLK;
        int32_t Mpre[BLK], Dv[BLK], H0[BLK], M[BLK], I[BLK];
        // X, Y: with one predecessor, its M and D at this block (for the records);
        // with several and TRACK, the record choices kept while the predecessors
        // are read: X = m1 | m4 << 16 (first predecessors, in priority order,
        // reaching the diagonal maximum), Y = dopen | dext << 16 (the vertical
        // maximum); 511 = none
        uint32_t X[BLK], Y[BLK];
        int32_t cmprev = NEG_INF;
        bool c_blk = false, c_prev = false, slow = !TRACK, slow0 = false;
        uint32_t hm = 0;  // bit l: Mpre[l] >= Dv[l], then (after the scan) M[l] == Mpre[l]
        uint32_t qlo = 0x04040404u, qhi = 0x04040404u;
        const uint32_t xinit = (TRACK && d >= 2) ? 0x01ff01ffu : (uint32_t)NEG_INF;
#pragma unroll
        for (int l = 0; l < BLK; l++) { Mpre[l] = NEG_INF; Dv[l] = NEG_INF; X[l] = Y[l] = xinit; }
        if (act) {
            const uint2 qw = *reinterpret_cast<const uint2*>(qsm + B * BLK);
            qlo = qw.x;
            qhi = qw.y;
            if (i == 0 && b == 0) Mpre[0] = 0;
            for (int k = 0; k < d; k++) {
                int pbsbe, pst, pbase;
                if (k == 0) { pbsbe = cur.pbsbe; pst = cur.pst; pbase = cur.pbase; }
                else { const int4 er = er_base[cur.e0 + k]; pbsbe = er.x; pst = er.y; pbase = er.w & 255; }
                const int pBs = pbsbe & 0xffff, pBe = pbsbe >> 16;
                const int32_t* src = blk_src(ring, a.rs, RB, pst);
                const PredMask mk = pred_mask(B, pBs, pBe);
                int32_t Mb[BLK], Db[BLK];
                int32_t mprev = NEG_INF;
                if (mk.prev_in) mprev = src[(B - 1 - pBs) * 16 + 7];
                if (mk.blk_in) {
                    load_block16(src + (B - pBs) * 16, Mb, Db);
                    if (TRACK && d >= 2) {
                        // the maxima of pass1_pred, keeping the first predecessor (in
                        // priority order) that reaches each final maximum
                        const int4 erk = er_base[cur.e0 + k];
                        const uint32_t pos = (uint32_t)erk.z >> 16;
                        const uint32_t m1v = (erk.w & 256) ? pos : 510u;
#pragma unroll
                        for (int l = 0; l < BLK; l++) {
                            const int32_t co = add32(Mb[l], sc.o1), ce = add32(Db[l], sc.e1);
                            const int32_t nd = mx(Dv[l], mx(co, ce));
                            if (nd > Dv[l]) {
                                Y[l] = (co == nd ? pos : 511u) | ((ce == nd ? pos : 511u) << 16);
                            } else {
                                if ((Y[l] & 0xffffu) == 511u && co == nd) Y[l] = (Y[l] & 0xffff0000u) | pos;
                                if ((Y[l] >> 16) == 511u && ce == nd) Y[l] = (Y[l] & 0xffffu) | (pos << 16);
                            }
                            Dv[l] = nd;
                        }
                        if (mk.diag) {
#pragma unroll
                            for (int l = 0; l < BLK; l++) {
                                const int qc = (int)(((l < 4 ? qlo : qhi) >> (8 * (l & 3))) & 255);
                                const bool bm = pbase == qc;
                                const int32_t src0 = l == 0 ? (b == 0 ? NEG_INF : mprev) : Mb[l > 0 ? l - 1 : 0];
                                const int32_t cand = add32(src0, bm ? sc.match : sc.mismatch);
                                const bool tracked = l > 0 || b != 0;  // the backtrack tests this same value
                                if (cand > Mpre[l]) {
                                    X[l] = tracked ? ((bm ? m1v : 511u) | (pos << 16)) : 0x01ff01ffu;
                                } else if (tracked && cand == Mpre[l]) {
                                    if ((X[l] >> 16) == 511u) X[l] = (X[l] & 0xffffu) | (pos << 16);
                                    if (bm && (X[l] & 0xffffu) == 511u) X[l] = (X[l] & 0xffff0000u) | m1v;
                                }
                                Mpre[l] = mx(Mpre[l], cand);
                            }
                        }
                    } else {
                        uint8_t qc8[BLK];
#pragma unroll
                        for (int l = 0; l < 4; l++) { qc8[l] = (uint8_t)(qlo >> (8 * l)); qc8[4 + l] = (uint8_t)(qhi >> (8 * l)); }
                        pass1_pred(sc, mk, b == 0, pbase, Mb, Db, mprev, qc8, Mpre, Dv);
                        if (d == 1) {
#pragma unroll
                            for (int l = 0; l < BLK; l++) { X[l] = (uint32_t)Mb[l]; Y[l] = (uint32_t)Db[l]; }
                        }
                    }
                }
                // where the backtrack's predecessor test and the fill's block-granular
                // diagonal differ (a predecessor's band starting in this block, or ending
                // just before it, or the row's first block), the choices are redone with
                // the backtrack's own test: the whole block in the first case, cell 0 else
                if (TRACK && d >= 2) {
                    slow |= mk.blk_in && !mk.diag;
                    slow0 |= mk.prev_in && !(mk.blk_in && mk.diag && b != 0);
                }
                if (d == 1) { cmprev = mprev; c_blk = mk.blk_in; c_prev = mk.prev_in; }
            }
        }
        // prefix max of the scan keys across the warp
        int32_t agg = INT_MIN;
#pragma unroll
        for (int l = 0; l < BLK; l++) {
            H0[l] = mx(Mpre[l], Dv[l]);
            if (TRACK && Mpre[l] >= Dv[l]) hm |= 1u << l;
            agg = mx(agg, add32(H0[l], -(j0 + l) * sc.e1));
        }
        if (!act) agg = INT_MIN;
        const int32_t incl = warp_incl_max(agg);
        int32_t P = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) P = INT_MIN;
        P = mx(P, carryP);
        const int32_t chunk_total = __shfl_sync(0xffffffffu, incl, 31);
        if (i == 0) {
#pragma unroll
            for (int l = 0; l < BLK; l++) { M[l] = H0[l]; I[l] = NEG_INF; }
        } else {
            int32_t run = P;
#pragma unroll
            for (int l = 0; l < BLK; l++) {
                I[l] = add32(sc.o1 + (j0 + l - 1) * sc.e1, run);
                M[l] = mx(H0[l], I[l]);
                if (TRACK && H0[l] < I[l]) hm &= ~(1u << l);
                run = mx(run, add32(H0[l], -(j0 + l) * sc.e1));
            }
        }
        if (ARGMAX && act) {
#pragma unroll
            for (int l = 0; l < BLK; l++)
                if (M[l] > bestM) { bestM = M[l]; bestJ = j0 + l; }  // first maximum of the row
        }
        const int32_t upM = __shfl_up_sync(0xffffffffu, M[BLK - 1], 1);
        const int32_t upI = __shfl_up_sync(0xffffffffu, I[BLK - 1], 1);
        const int32_t Ml0 = lane > 0 ? upM : carryM, Il0 = lane > 0 ? upI : carryI;
        const int32_t nextM = __shfl_sync(0xffffffffu, M[BLK - 1], 31);
        const int32_t nextI = __shfl_sync(0xffffffffu, I[BLK - 1], 31);
        if (act) {
            if (d <= 1) {
                uint32_t lo = 0, hi = 0;
#pragma unroll
                for (int l = 0; l < BLK; l++) {
                    const int32_t Ml = l > 0 ? M[l - 1] : Ml0, Il = l > 0 ? I[l - 1] : Il0;
                    uint32_t r = own_flags(sc, j0 + l, M[l], Dv[l], I[l], Ml, Il);
                    if (d == 1) {
                        const int qc = (int)(((l < 4 ? qlo : qhi) >> (8 * (l & 3))) & 255);
                        const bool inr = l == 0 ? c_prev : c_blk;
                        const int32_t mv = l == 0 ? cmprev : (int32_t)X[l > 0 ? l - 1 : 0];
                        const bool bm = cur.pbase == qc;
                        const bool eqM = inr && M[l] == add32(mv, bm ? sc.match : sc.mismatch);
                        if (eqM) r |= R_M4;
                        if (eqM && bm && cur.w1ok) r |= R_M1;
                        if (c_blk && Dv[l] == add32((int32_t)X[l], sc.o1)) r |= R_DOPEN;
                        else if (c_blk && Dv[l] == add32((int32_t)Y[l], sc.e1)) r |= R_DEXT;
                    }
                    if (l < 4) lo |= r << (8 * l);
                    else hi |= r << (8 * (l - 4));
                }
                *reinterpret_cast<uint2*>(a.tb + cur.tb + b * BLK) = make_uint2(lo, hi);
            } else {
                // choices per cell: m1 | m4 << 16, dopen | dext << 16 (511 = none,
                // 510 = the best matching predecessor failed the weight threshold)
                uint32_t* cm = X;
                uint32_t* cd = Y;
                if (!slow) {
                    // tracked choices stand where M is the diagonal maximum itself
#pragma unroll
                    for (int l = 0; l < BLK; l++)
                        if (!((hm >> l) & 1u)) cm[l] = 0x01ff01ffu;
                    if (slow0) {
                        // cell 0 by the backtrack's own test, over every predecessor
                        uint32_t c0 = 0x01ff01ffu;
                        const int qc = (int)(qlo & 255u);
                        for (int k = 0; k < d; k++) {
                            const int4 er = er_base[cur.e0 + k];
                            const int pBs = er.x & 0xffff, pBe = er.x >> 16;
                            if (!(B - 1 >= pBs && B - 1 <= pBe - 2)) continue;  // prev_in
                            const int32_t mv = blk_src(ring, a.rs, RB, er.y)[(B - 1 - pBs) * 16 + 7];
                            const uint32_t pos = (uint32_t)er.z >> 16;
                            const bool bm = (er.w & 255) == qc;
                            if (M[0] != add32(mv, bm ? sc.match : sc.mismatch)) continue;
                            if ((c0 >> 16) == 511u) c0 = (c0 & 0xffffu) | (pos << 16);
                            if (bm && (c0 & 0xffffu) == 511u) c0 = (c0 & 0xffff0000u) | ((er.w & 256) ? pos : 510u);
                        }
                        cm[0] = c0;
                    }
                }
#pragma unroll
                for (int l = 0; l < BLK; l++)
                    if (slow) { cm[l] = 0x01ff01ffu; cd[l] = 0x01ff01ffu; }
                for (int k = 0; k < (slow ? d : 0); k++) {
                    const int4 er = er_base[cur.e0 + k];
                    const int pBs = er.x & 0xffff, pBe = er.x >> 16;
                    const int32_t* src = blk_src(ring, a.rs, RB, er.y);
                    const PredMask mk = pred_mask(B, pBs, pBe);
                    if (!(mk.blk_in || mk.prev_in)) continue;
                    const uint32_t pos = (uint32_t)er.z >> 16;
                    const int pbase = er.w & 255;
                    const uint32_t m1v = (er.w & 256) ? pos : 510u;
                    int32_t Mb[BLK], Db[BLK];
                    int32_t mprev = NEG_INF;
                    if (mk.prev_in) mprev = src[(B - 1 - pBs) * 16 + 7];
                    if (mk.blk_in) load_block16(src + (B - pBs) * 16, Mb, Db);
                    else {
#pragma unroll
                        for (int l = 0; l < BLK; l++) Mb[l] = Db[l] = NEG_INF;
                    }
#pragma unroll
                    for (int l = 0; l < BLK; l++) {
                        const int qc = (int)(((l < 4 ? qlo : qhi) >> (8 * (l & 3))) & 255);
                        const bool inr = l == 0 ? mk.prev_in : mk.blk_in;
                        const int32_t mv = l == 0 ? mprev : Mb[l > 0 ? l - 1 : 0];
                        const bool bm = pbase == qc;
                        const bool eqM = inr && M[l] == add32(mv, bm ? sc.match : sc.mismatch);
                        if (eqM && (cm[l] >> 16) == 511u) cm[l] = (cm[l] & 0xffffu) | (pos << 16);
                        if (eqM && bm && (cm[l] & 0xffffu) == 511u) cm[l] = (cm[l] & 0xffff0000u) | m1v;
                        if (mk.blk_in) {
                            if ((cd[l] & 0xffffu) == 511u && Dv[l] == add32(Mb[l], sc.o1))
                                cd[l] = (cd[l] & 0xffff0000u) | pos;
                            if ((cd[l] >> 16) == 511u && Dv[l] == add32(Db[l], sc.e1))
                                cd[l] = (cd[l] & 0xffffu) | (pos << 16);
                        }
                    }
                }
                uint32_t r[BLK];
#pragma unroll
                for (int l = 0; l < BLK; l++) {
                    const int32_t Ml = l > 0 ? M[l - 1] : Ml0, Il = l > 0 ? I[l - 1] : Il0;
                    uint32_t w = own_flags(sc, j0 + l, M[l], Dv[l], I[l], Ml, Il) & 15u;
                    uint32_t m1 = cm[l] & 0xffffu, m4 = cm[l] >> 16;
                    if (m1 == 510u) m1 = W_NONE;
                    uint32_t dd = cd[l] & 0xffffu;
                    if (dd == 511u) {
                        dd = cd[l] >> 16;
                        if (dd != 511u) w |= W_DEXT;
                    }
                    r[l] = w | (m1 << W_M1_SHIFT) | (m4 << W_M4_SHIFT) | (dd << W_D_SHIFT);
                }
                uint4* tdst = reinterpret_cast<uint4*>(a.tb + cur.tb + b * BLK * 4);
                tdst[0] = make_uint4(r[0], r[1], r[2], r[3]);
                tdst[1] = make_uint4(r[4], r[5], r[6], r[7]);
            }
            store_block16(dst + b * 16, M, Dv);
        }
        carryP = mx(carryP, chunk_total);
        carryM = nextM;
        carryI = nextI;
    }
}

// One row of the adaptive / full-band warp fill (dp_fill_warp_dyn): the chunk
// loop of fill_row, with the predecessors' records `er` (backtrack priority
// order, bands and row-store locations patched in) read once per chunk, and
// the record choices of multi-predecessor rows kept in one pass
// (dp_core.h track_d / track_m): per cell the running maximum of each kind
// of term plus a 4-bit first position per choice, folded into one 16-bit
// word (z) as soon as the predecessors are read:
//   z bits 0..3 D choice (dopen, else dext; 15 none), bit 4 W_DEXT,
//          8..11 m4, 12..15 m1 (15 none; gated by M == Mpre at the record).
// Register roles by row kind: with one predecessor Mpre / Dv are the
// diagonal / vertical maxima and pa / pb copies of its M / D block (for the
// 1-byte records); with several, Mpre is the diagonal maximum, Dv the
// maximum of M_p + o1, pb of D_p + e1 and pa of the matching diagonal terms
// until the pass ends, when Dv becomes the vertical maximum.
// Rows with more than TRACK_MAX_D predecessors, and blocks where the fill's
// block-granular masks differ from the backtrack's per-cell test, take the
// second pass over the predecessors (as fill_row does).
template <bool ARGMAX>
__device__ __forceinline__ void fill_row_dyn(const DpArgs& a, const RowDesc& cur, const int4* __restrict__ er,
                                             const uint8_t* __restrict__ qsm, int i, int lane, int32_t& bestM,
                                             int& bestJ) {
    const Scoring sc = a.sc;
    const int32_t K = add32(add32(NEG_INF, sc.e1), -sc.o1);
    const int Bs = cur.bsbe & 0xffff, Be = cur.bsbe >> 16, bn = Be - Bs - 1;
    const int d = cur.d;
    const bool multi = d >= 2;
    int32_t* dst = a.rs + cur.st;
    const int nch = (bn + 31) >> 5;
    int32_t carryP = K, carryM = NEG_INF, carryI = NEG_INF;
    for (int c = 0; c < nch; c++) {
        const int b = c * 32 + lane;
        const bool act = b < bn;
        const int B = Bs + b;
        const int j0 = b * BLK;
        int32_t Mpre[BLK], Dv[BLK], H0[BLK], M[BLK], I[BLK];
        int32_t pa[BLK], pb[BLK];
        uint32_t z2[BLK / 2];  // choice words: cell 2t in bits 0..15, cell 2t+1 in bits 16..31
        int32_t cmprev = NEG_INF;
        bool c_blk = false, c_prev = false, slow = d > TRACK_MAX_D, slow0 = false;
        uint32_t f1lo = 0, f1hi = 0, m1lo = 0, m1hi = 0;  // one predecessor: record flags, see below
        uint32_t hm = 0;  // bit l: Mpre[l] >= Dv[l], then (after the scan) M[l] == Mpre[l]
        uint32_t qlo = 0x04040404u, qhi = 0x04040404u;
        const int32_t minit = multi ? INT_MIN : NEG_INF;
#pragma unroll
        for (int l = 0; l < BLK; l++) Mpre[l] = Dv[l] = pa[l] = pb[l] = minit;
#pragma unroll
        for (int t = 0; t < BLK / 2; t++) z2[t] = 0xffffffffu;
        if (act) {
            const uint2 qw = *reinterpret_cast<const uint2*>(qsm + B * BLK);
            qlo = qw.x;
            qhi = qw.y;
            if (i == 0 && b == 0) Mpre[0] = 0;
        }
        auto qc_at = [&](int l) { return (int)(((l < 4 ? qlo : qhi) >> (8 * (l & 3))) & 255u); };
        if (act) {
            for (int k = 0; k < d; k++) {
                const int4 ek = er[k];
                const int pBs = ek.x & 0xffff, pBe = ek.x >> 16;
                const int32_t* src = a.rs + ek.y;
                const int pbase = ek.w & 255;
                const PredMask mk = pred_mask(B, pBs, pBe);
                int32_t mprev = NEG_INF;
                if (mk.prev_in) mprev = src[(B - 1 - pBs) * 16 + 7];
                if (mk.blk_in) {
                    int32_t Mb[BLK], Db[BLK];
                    load_block16(src + (B - pBs) * 16, Mb, Db);
                    if (multi) {
                        const uint32_t pos = ((uint32_t)ek.z >> 16) & 15u;  // exact when d <= TRACK_MAX_D
                        const uint32_t p1 = (ek.w & 256) ? pos : Y_NONE;
#pragma unroll
                        for (int l = 0; l < BLK; l++)
                            track_d(sc, Mb[l], Db[l], pos, Dv[l], pb[l], z2[l >> 1], 16 * (l & 1));
                        if (mk.diag) {
                            // cell 0 of the row's first block reads NEG_INF (the lane quirk); the
                            // backtrack never takes that term, so it records no position
                            const bool first = b == 0;
                            const bool bm0 = pbase == qc_at(0);
                            track_m(add32(first ? NEG_INF : mprev, bm0 ? sc.match : sc.mismatch), bm0,
                                    first ? Y_NONE : pos, first ? Y_NONE : p1, Mpre[0], pa[0], z2[0], 0);
#pragma unroll
                            for (int l = 1; l < BLK; l++) {
                                const bool bm = pbase == qc_at(l);
                                track_m(add32(Mb[l - 1], bm ? sc.match : sc.mismatch), bm, pos, p1, Mpre[l], pa[l],
                                        z2[l >> 1], 16 * (l & 1));
                            }
                        }
                    } else {
                        // one predecessor: its terms and, while they are in registers, the
                        // 1-byte record's predecessor flags (byte l of f1lo / f1hi): the
                        // vertical choice (the fill's and the backtrack's vertical tests are
                        // the same block test) and the diagonal one, which stands when
                        // M == Mpre (checked after the scan) wherever the fill's diagonal
                        // mask matches the backtrack's per-cell test (else slow: recomputed)
#pragma unroll
                        for (int l = 0; l < BLK; l++) {
                            const int32_t ce = add32(Db[l], sc.e1), co = add32(Mb[l], sc.o1);
                            const int32_t dv = mx(mx(NEG_INF, ce), co);
                            Dv[l] = dv;
                            const uint32_t fd = co == dv ? R_DOPEN : (ce == dv ? R_DEXT : 0u);
                            if (l < 4) f1lo |= fd << (8 * l);
                            else f1hi |= fd << (8 * (l - 4));
                        }
                        if (mk.diag) {
#pragma unroll
                            for (int l = 0; l < BLK; l++) {
                                const bool bm = pbase == qc_at(l);
                                const int32_t src0 = l == 0 ? (b == 0 ? NEG_INF : mprev) : Mb[l > 0 ? l - 1 : 0];
                                const int32_t cand = add32(src0, bm ? sc.match : sc.mismatch);
                                const int32_t mp = mx(NEG_INF, cand);
                                Mpre[l] = mp;
                                // cell 0 counts only where the backtrack tests the same value
                                const bool tested = l > 0 || (mk.prev_in && b != 0);
                                const uint32_t fm = (tested && cand == mp) ? (R_M4 | ((bm && cur.w1ok) ? R_M1 : 0u)) : 0u;
                                if (l < 4) m1lo |= fm << (8 * l);
                                else m1hi |= fm << (8 * (l - 4));
                            }
                        }
                    }
                }
                if (multi) {
                    slow |= mk.blk_in && !mk.diag;
                    slow0 |= mk.prev_in && !(mk.blk_in && mk.diag && b != 0);
                } else {
                    cmprev = mprev; c_blk = mk.blk_in; c_prev = mk.prev_in;
                    slow |= (mk.blk_in && !mk.diag) || (mk.prev_in && !(mk.blk_in && mk.diag && b != 0));
                }
            }
        }
        if (multi) {
            // final maxima, and the choices folded into z (see above)
#pragma unroll
            for (int l = 0; l < BLK; l++) {
                const int sh = 16 * (l & 1);
                const uint32_t y = (z2[l >> 1] >> sh) & 0xffffu;
                const int32_t mp = mx(NEG_INF, Mpre[l]);
                const int32_t dv = mx(NEG_INF, mx(Dv[l], pb[l]));  // Dv: max of M_p + o1, pb: of D_p + e1
                const bool okO = Dv[l] == dv, okE = pb[l] == dv;
                uint32_t w = okO ? (y & 15u) : (okE ? (((y >> Y_E) & 15u) | W_DEXT) : Y_NONE);
                w |= Mpre[l] == mp ? (y & 0x0f00u) : 0x0f00u;
                w |= pa[l] == mp ? (y & 0xf000u) : 0xf000u;
                z2[l >> 1] = (z2[l >> 1] & ~(0xffffu << sh)) | (w << sh);
                Mpre[l] = mp;
                Dv[l] = dv;
            }
        }
        // prefix max of the scan keys across the warp
        int32_t agg = INT_MIN;
#pragma unroll
        for (int l = 0; l < BLK; l++) {
            H0[l] = mx(Mpre[l], Dv[l]);
            if (Mpre[l] >= Dv[l]) hm |= 1u << l;
            agg = mx(agg, add32(H0[l], -(j0 + l) * sc.e1));
        }
        if (!act) agg = INT_MIN;
        const int32_t incl = warp_incl_max(agg);
        int32_t P = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) P = INT_MIN;
        P = mx(P, carryP);
        const int32_t chunk_total = __shfl_sync(0xffffffffu, incl, 31);
        if (i == 0) {
#pragma unroll
            for (int l = 0; l < BLK; l++) { M[l] = H0[l]; I[l] = NEG_INF; }
        } else {
            int32_t run = P;
#pragma unroll
            for (int l = 0; l < BLK; l++) {
                I[l] = add32(sc.o1 + (j0 + l - 1) * sc.e1, run);
                M[l] = mx(H0[l], I[l]);
                if (H0[l] < I[l]) hm &= ~(1u << l);
                run = mx(run, add32(H0[l], -(j0 + l) * sc.e1));
            }
        }
        if (ARGMAX && act) {
#pragma unroll
            for (int l = 0; l < BLK; l++)
                if (M[l] > bestM) { bestM = M[l]; bestJ = j0 + l; }  // first maximum of the row
        }
        const int32_t upM = __shfl_up_sync(0xffffffffu, M[BLK - 1], 1);
        const int32_t upI = __shfl_up_sync(0xffffffffu, I[BLK - 1], 1);
        const int32_t Ml0 = lane > 0 ? upM : carryM, Il0 = lane > 0 ? upI : carryI;
        const int32_t nextM = __shfl_sync(0xffffffffu, M[BLK - 1], 31);
        const int32_t nextI = __shfl_sync(0xffffffffu, I[BLK - 1], 31);
        if (act) {
            if (!multi) {
                uint32_t lo = 0, hi = 0;
#pragma unroll
                for (int l = 0; l < BLK; l++) {
                    const int32_t Ml = l > 0 ? M[l - 1] : Ml0, Il = l > 0 ? I[l - 1] : Il0;
                    const uint32_t r = own_flags(sc, j0 + l, M[l], Dv[l], I[l], Ml, Il);
                    if (l < 4) lo |= r << (8 * l);
                    else hi |= r << (8 * (l - 4));
                }
                if (d == 1) {
                    // the diagonal flags stand in cells where M == Mpre (byte mask of hm)
                    const uint32_t hlo = ((hm & 15u) * 0x00204081u & 0x01010101u) * 0xffu;
                    const uint32_t hhi = ((hm >> 4) * 0x00204081u & 0x01010101u) * 0xffu;
                    lo |= f1lo | (m1lo & hlo);
                    hi |= f1hi | (m1hi & hhi);
                    if (slow) {
                        // a block where the fill's diagonal mask and the backtrack's per-cell
                        // test differ: the diagonal flags by the backtrack's own test
                        const int pBs = cur.pbsbe & 0xffff;
                        const int32_t* src = a.rs + cur.pst;
                        int32_t Mb[BLK];
#pragma unroll
                        for (int l = 0; l < BLK; l++) Mb[l] = NEG_INF;
                        if (c_blk) {
                            const int4* q = reinterpret_cast<const int4*>(src + (B - pBs) * 16);
                            const int4 u = q[0], v = q[1];
                            Mb[0] = u.x; Mb[1] = u.y; Mb[2] = u.z; Mb[3] = u.w;
                            Mb[4] = v.x; Mb[5] = v.y; Mb[6] = v.z; Mb[7] = v.w;
                        }
                        lo &= ~0x30303030u;
                        hi &= ~0x30303030u;
#pragma unroll
                        for (int l = 0; l < BLK; l++) {
                            const bool inr = l == 0 ? c_prev : c_blk;
                            const int32_t mv = l == 0 ? cmprev : Mb[l > 0 ? l - 1 : 0];
                            const bool bm = cur.pbase == qc_at(l);
                            const bool eqM = inr && M[l] == add32(mv, bm ? sc.match : sc.mismatch);
                            const uint32_t fm = eqM ? (R_M4 | ((bm && cur.w1ok) ? R_M1 : 0u)) : 0u;
                            if (l < 4) lo |= fm << (8 * l);
                            else hi |= fm << (8 * (l - 4));
                        }
                    }
                }
                *reinterpret_cast<uint2*>(a.tb + cur.tb + b * BLK) = make_uint2(lo, hi);
            } else {
                uint32_t r[BLK];
                if (!slow) {
                    uint32_t c0 = 0x01ff01ffu;
                    if (slow0) {
                        // cell 0 by the backtrack's own test, over every predecessor
                        const int qc = qc_at(0);
                        for (int k = 0; k < d; k++) {
                            const int4 ek = er[k];
                            const int pBs = ek.x & 0xffff, pBe = ek.x >> 16;
                            if (!(B - 1 >= pBs && B - 1 <= pBe - 2)) continue;  // prev_in
                            const int32_t mv = a.rs[ek.y + (B - 1 - pBs) * 16 + 7];
                            const uint32_t pos = (uint32_t)ek.z >> 16;
                            const bool bm = (ek.w & 255) == qc;
                            if (M[0] != add32(mv, bm ? sc.match : sc.mismatch)) continue;
                            if ((c0 >> 16) == 511u) c0 = (c0 & 0xffffu) | (pos << 16);
                            if (bm && (c0 & 0xffffu) == 511u) c0 = (c0 & 0xffff0000u) | ((ek.w & 256) ? pos : 510u);
                        }
                    }
#pragma unroll
                    for (int l = 0; l < BLK; l++) {
                        const int32_t Ml = l > 0 ? M[l - 1] : Ml0, Il = l > 0 ? I[l - 1] : Il0;
                        const uint32_t own = own_flags(sc, j0 + l, M[l], Dv[l], I[l], Ml, Il) & 15u;
                        const uint32_t w = (z2[l >> 1] >> (16 * (l & 1))) & 0xffffu;
                        const bool h = (hm >> l) & 1u;
                        const uint32_t n4 = (w >> Y_4) & 15u, n1 = (w >> Y_1) & 15u, nd = w & 15u;
                        uint32_t m4 = (h && n4 != Y_NONE) ? n4 : W_NONE;
                        uint32_t m1 = (h && n1 != Y_NONE) ? n1 : W_NONE;
                        if (l == 0 && slow0) {
                            m1 = c0 & 0xffffu;
                            if (m1 == 510u) m1 = W_NONE;
                            m4 = c0 >> 16;
                        }
                        const uint32_t dd = nd != Y_NONE ? nd : W_NONE;
                        r[l] = own | (w & W_DEXT) | (m1 << W_M1_SHIFT) | (m4 << W_M4_SHIFT) | (dd << W_D_SHIFT);
                    }
                } else {
                    // the diagonal choices by the backtrack's own test, over every predecessor;
                    // the vertical choices in z stand (the fill's and the backtrack's vertical
                    // tests are the same block test) unless the row has more predecessors
                    // than z's 4-bit positions hold
                    const bool dwide = d > TRACK_MAX_D;
                    uint32_t cm[BLK], cd[BLK];
#pragma unroll
                    for (int l = 0; l < BLK; l++) cm[l] = cd[l] = 0x01ff01ffu;
                    for (int k = 0; k < d; k++) {
                        const int4 ek = er[k];
                        const int pBs = ek.x & 0xffff, pBe = ek.x >> 16;
                        const int32_t* src = a.rs + ek.y;
                        const PredMask mk = pred_mask(B, pBs, pBe);
                        if (!(mk.blk_in || mk.prev_in)) continue;
                        const uint32_t pos = (uint32_t)ek.z >> 16;
                        const int pbase = ek.w & 255;
                        const uint32_t m1v = (ek.w & 256) ? pos : 510u;
                        int32_t Mb[BLK];
                        int32_t mprev = NEG_INF;
                        if (mk.prev_in) mprev = src[(B - 1 - pBs) * 16 + 7];
                        if (mk.blk_in) {
                            const int4* q = reinterpret_cast<const int4*>(src + (B - pBs) * 16);
                            const int4 u = q[0], v = q[1];
                            Mb[0] = u.x; Mb[1] = u.y; Mb[2] = u.z; Mb[3] = u.w;
                            Mb[4] = v.x; Mb[5] = v.y; Mb[6] = v.z; Mb[7] = v.w;
                            if (dwide) {
                                const int4 x = q[2], y = q[3];
                                const int32_t Db[BLK] = {x.x, x.y, x.z, x.w, y.x, y.y, y.z, y.w};
#pragma unroll
                                for (int l = 0; l < BLK; l++) {
                                    if ((cd[l] & 0xffffu) == 511u && Dv[l] == add32(Mb[l], sc.o1))
                                        cd[l] = (cd[l] & 0xffff0000u) | pos;
                                    if ((cd[l] >> 16) == 511u && Dv[l] == add32(Db[l], sc.e1))
                                        cd[l] = (cd[l] & 0xffffu) | (pos << 16);
                                }
                            }
                        } else {
#pragma unroll
                            for (int l = 0; l < BLK; l++) Mb[l] = NEG_INF;
                        }
#pragma unroll
                        for (int l = 0; l < BLK; l++) {
                            const bool inr = l == 0 ? mk.prev_in : mk.blk_in;
                            const int32_t mv = l == 0 ? mprev : Mb[l > 0 ? l - 1 : 0];
                            const bool bm = pbase == qc_at(l);
                            const bool eqM = inr && M[l] == add32(mv, bm ? sc.match : sc.mismatch);
                            if (eqM && (cm[l] >> 16) == 511u) cm[l] = (cm[l] & 0xffffu) | (pos << 16);
                            if (eqM && bm && (cm[l] & 0xffffu) == 511u) cm[l] = (cm[l] & 0xffff0000u) | m1v;
                        }
                    }
#pragma unroll
                    for (int l = 0; l < BLK; l++) {
                        const int32_t Ml = l > 0 ? M[l - 1] : Ml0, Il = l > 0 ? I[l - 1] : Il0;
                        const uint32_t own = own_flags(sc, j0 + l, M[l], Dv[l], I[l], Ml, Il) & 15u;
                        const uint32_t w = (z2[l >> 1] >> (16 * (l & 1))) & 0xffffu;
                        uint32_t m1 = cm[l] & 0xffffu;
                        if (m1 == 510u) m1 = W_NONE;
                        const uint32_t m4 = cm[l] >> 16, nd = w & 15u;
                        uint32_t dd = nd != Y_NONE ? nd : W_NONE, dext = w & W_DEXT;
                        if (dwide) {
                            dd = cd[l] & 0xffffu;
                            dext = 0;
                            if (dd == 511u) {
                                dd = cd[l] >> 16;
                                if (dd != 511u) dext = W_DEXT;
                            }
                        }
                        r[l] = own | dext | (m1 << W_M1_SHIFT) | (m4 << W_M4_SHIFT) | (dd << W_D_SHIFT);
                    }
                }
                uint4* tdst = reinterpret_cast<uint4*>(a.tb + cur.tb + b * BLK * 4);
                tdst[0] = make_uint4(r[0], r[1], r[2], r[3]);
                tdst[1] = make_uint4(r[4], r[5], r[6], r[7]);
            }
            store_block16(dst + b * 16, M, Dv);
        }
        carryP = mx(carryP, chunk_total);
        carryM = nextM;
        carryI = nextI;
    }
}

__device__ void dp_fill_warp_static(const DpArgs& a, const RowDesc* __restrict__ desc, const int4* __restrict__ erec,
                                    int32_t* ring, int RB, const uint8_t* qsm, unsigned char* stage, int lane) {
    const int n = a.v.n, m = a.qlen + 1;
    const Scoring sc = a.sc;
    const int32_t K = add32(add32(NEG_INF, sc.e1), -sc.o1);
    RowDesc* sdesc = reinterpret_cast<RowDesc*>(stage);
    int4* serec = reinterpret_cast<int4*>(stage + STAGE_ROWS * sizeof(RowDesc));
    int64_t cells = 0, ecells = 0;
    for (int i0 = 0; i0 < n; i0 += STAGE_ROWS) {
        const int cnt = min(STAGE_ROWS, n - i0);
        // stage: descriptors of rows i0.., and their predecessor records when they fit
        __syncwarp();
        {
            const int4* src = reinterpret_cast<const int4*>(desc + i0);
            for (int x = lane; x < cnt * 3; x += 32) reinterpret_cast<int4*>(sdesc)[x] = src[x];
        }
        __syncwarp();
        const int e_lo = sdesc[0].e0;
        const int e_hi = sdesc[cnt - 1].e0 + sdesc[cnt - 1].d;
        const bool staged = e_hi - e_lo <= STAGE_EDGES;
        if (staged)
            for (int e = lane; e < e_hi - e_lo; e += 32) serec[e] = erec[e_lo + e];
        __syncwarp();
        const int4* er_base = staged ? serec - e_lo : erec;
        for (int i = i0; i < i0 + cnt; i++) {
            const RowDesc cur = sdesc[i - i0];
            const int64_t rc = (int64_t)((cur.bsbe >> 16) - (cur.bsbe & 0xffff) - 1) * BLK;
            cells += rc;
            ecells += rc * cur.d;
            int32_t bm = 0;
            int bj = 0;
            fill_row<false, false>(a, cur, er_base, ring, RB, qsm, i, lane, bm, bj);
            __syncwarp();
        }
    }
    if (lane == 0) {
        const RowMeta last = a.meta[n - 1];
        const int jm = m - last.Bs * BLK;
        const int32_t* src = blk_src(ring, a.rs, RB, (int)last.st);
        a.out[1] = src[(jm / BLK) * 16 + jm % BLK];
        a.out[3] = (int32_t)(cells > INT_MAX ? INT_MAX : cells);
        a.out[6] = (int32_t)(ecells > INT_MAX ? INT_MAX : ecells);
        a.out[0] = ST_OK;
    }
    __syncwarp();
}

// Warp fill for bands known only row by row (adaptive band, -B; or the full
// band, f = 0): the same chunk loop and records as the static fill
// (fill_row), with each row's descriptor assembled when the row is reached:
// its band from the adaptive state (row_band), its row-store location (a
// full-width ring of ring_rows rows in the slot; rows with a successor
// ring_rows or more rows ahead go to the spill area), its record offset (a
// running sum), and its predecessor records with the predecessors' bands
// and locations (staged in shared memory). After an adaptive row the warp
// finds the first maximum of M and lane 0 updates the adaptive state
// (src/align.cpp:1516-1568). out[4] / out[5]: record bytes and spilled
// row-store entries used.
constexpr int DYN_STAGE_EDGES = 128;
__device__ void dp_fill_warp_dyn(const DpArgs& a, int4* __restrict__ erec, const int32_t* __restrict__ vmaxs,
                                 const uint8_t* __restrict__ qsm, int4* sed, int32_t* upd, int lane) {
    const int n = a.v.n, m = a.qlen + 1;
    const bool adaptive = a.f > 0 && a.ab_band;
    if (adaptive)
        for (int r = lane; r < n; r += 32) adaptive_init_entry(a, r, m);
    __syncwarp();
    const int64_t ring_part = (int64_t)a.ring_rows * a.ring_blocks * 16;
    int64_t st_next = ring_part, tb_next = 0, cells = 0, ecells = 0;
    for (int i = 0; i < n; i++) {
        int Bs, Be;
        row_band(a, i, m, Bs, Be);
        if (i == 0) Bs = 0;
        const int bn = Be - Bs - 1;
        const int e0 = a.v.in_ptr[i];
        const int d = i == 0 ? 0 : a.v.in_ptr[i + 1] - e0;
        const int bpc = d >= 2 ? 4 : 1;
        const bool spill = a.ring_rows <= 0 || (vmaxs[i] - i >= a.ring_rows) || bn > a.ring_blocks;
        const int64_t row_st = spill ? st_next : (int64_t)(i % a.ring_rows) * a.ring_blocks * 16;
        int st = ST_OK;
        if (bn < 0) st = ST_DEGENERATE;
        else if (d > MAX_MULTI_PRED) st = ST_INDEGREE;
        else if ((spill && row_st + (int64_t)bn * 16 > a.rs_cap) || tb_next + (int64_t)bn * BLK * bpc > a.tb_cap ||
                 row_st > INT_MAX || tb_next > INT_MAX)
            st = ST_OOM;
        if (st != ST_OK) {
            if (lane == 0) a.out[0] = st;
            __syncwarp();
            return;
        }
        if (spill) st_next = row_st + (int64_t)bn * 16;
        if (lane == 0) {
            RowMeta rm;
            rm.Bs = Bs; rm.Be = Be; rm.st = row_st; rm.tb = tb_next;
            a.meta[i] = rm;
        }
        // the adaptive update's inputs, copied while the row is filled
        int ns = 0, base_i = 0, hql = 0;
        bool pf = false;
        if (adaptive && i >= 1) {
            const int o0 = a.v.out_ptr[i];
            ns = a.v.out_ptr[i + 1] - o0;
            base_i = a.v.base[i];
            hql = a.v.hq_loc[i];
            pf = d <= 32 && ns <= 32;
            if (pf) {
                const int32_t* st_ = a.state;
                if (lane < ns) {
                    const int sr = a.v.out_row[o0 + lane];
                    upd[UPD_SROW + lane] = sr;
                    cp_async4(upd + UPD_SOL + lane, st_ + AB_OL * n + sr);
                    cp_async4(upd + UPD_SOR + lane, st_ + AB_OR * n + sr);
                    cp_async4(upd + UPD_SPL + lane, st_ + AB_PL * n + sr);
                    cp_async4(upd + UPD_SPR + lane, st_ + AB_PR * n + sr);
                    cp_async4(upd + UPD_SOW + lane, st_ + AB_OW * n + sr);
                }
                if (lane < 4) {
                    const int arr = lane == 0 ? AB_SL : lane == 1 ? AB_OW : lane == 2 ? AB_OL : AB_OR;
                    cp_async4(upd + UPD_OWN + lane, st_ + arr * n + i);
                }
            }
        }
        // predecessor records with the predecessors' bands and locations
        int4* er = d <= DYN_STAGE_EDGES ? sed : erec + e0;
        for (int k = lane; k < d; k += 32) {
            int4 rec = erec[e0 + k];
            if (pf) {
                cp_async4(upd + UPD_PSL + k, a.state + AB_SL * n + rec.x);
                cp_async4(upd + UPD_PMP + k, a.state + AB_MP * n + rec.x);
            }
            const RowMeta pm = a.meta[rec.x];
            rec.x = pm.Bs | (pm.Be << 16);
            rec.y = (int32_t)pm.st;
            er[k] = rec;
        }
        if (pf) cp_async_commit_all();
        __syncwarp();
        RowDesc cur;
        cur.bsbe = Bs | (Be << 16);
        cur.st = (int32_t)row_st;
        cur.tb = (int32_t)tb_next;
        cur.e0 = 0;
        cur.d = d;
        cur.ind = a.v.ind[i];
        if (d >= 1) {
            const int4 r0 = er[0];
            cur.pbsbe = r0.x; cur.pst = r0.y; cur.pbase = r0.w & 255; cur.pw = r0.z & 0xffff;
            cur.w1ok = (r0.w >> 8) & 1;
            cur.prow0 = 0;
        } else {
            cur.pbsbe = cur.pst = cur.pbase = cur.pw = cur.w1ok = cur.prow0 = 0;
        }
        int32_t bestM = INT_MIN;
        int bestJ = 0;
        if (adaptive) fill_row_dyn<true>(a, cur, er, qsm, i, lane, bestM, bestJ);
        else fill_row_dyn<false>(a, cur, er, qsm, i, lane, bestM, bestJ);
        cells += (int64_t)bn * BLK;
        ecells += (int64_t)bn * BLK * d;
        if (adaptive && i >= 1) {
            // first maximum of the row: largest M, then smallest column
            unsigned long long key = bestM == INT_MIN ? 0ull
                                     : ((unsigned long long)((uint32_t)bestM ^ 0x80000000u) << 32) |
                                           (unsigned long long)(0xffffffffu - (uint32_t)bestJ);
            key = warp_max_u64(key);
            const int max_j = bn > 0 ? (int)(0xffffffffu - (uint32_t)(key & 0xffffffffu)) : 0;
            if (pf) {
                cp_async_wait_all();
                __syncwarp();
                adaptive_update_pf(a, i, Bs, max_j, lane, upd, d, ns, base_i, hql, qsm);
            } else {
                adaptive_update_warp(a, i, Bs, max_j, lane);
            }
        }
        tb_next = (tb_next + (int64_t)bn * BLK * bpc + 15) & ~(int64_t)15;
        __syncwarp();
    }
    if (lane == 0) {
        const RowMeta last = a.meta[n - 1];
        const int jm = m - last.Bs * BLK;
        a.out[1] = a.rs[last.st + (int64_t)(jm / BLK) * 16 + jm % BLK];
        a.out[3] = (int32_t)(cells > INT_MAX ? INT_MAX : cells);
        a.out[6] = (int32_t)(ecells > INT_MAX ? INT_MAX : ecells);
        a.out[4] = (int32_t)tb_next;
        a.out[5] = (int32_t)(st_next - ring_part);
        a.out[0] = ST_OK;
    }
    __syncwarp();
}

// Backtrack over the records (src/align.cpp:1572-1736, same decisions as
// backtrack_records) with the whole warp. The path mostly steps
// (i, j) -> (i-1, j-1), so lane k preloads the descriptor of row i-k and its
// record at column acj-k; the walk consumes lane t's values through shuffles
// while the path stays on that diagonal and preloads again from wherever it
// leaves it. All lanes run the walk (uniform control flow); lane 0 stores
// the moves.
__device__ int bt_warp_static(const RowDesc* __restrict__ desc, const int32_t* __restrict__ in_row,
                              const uint8_t* __restrict__ in_base, const uint8_t* __restrict__ tb,
                              const uint8_t* __restrict__ qs, int n, int m, int32_t* moves, int moves_cap,
                              int32_t& nm_out, int lane) {
    int i = n - 1, acj = m, op = ALL_OP, nm = 0;
    int status = ST_OK;
    while ((i > 0 || acj > 0) && status == ST_OK) {
        const int i0 = i, a0 = acj;
        // preload: lane k -> (i0 - k, a0 - k)
        const int ri = i0 - lane, cj = a0 - lane;
        int bsbe = 0, d = 0;
        uint32_t rec = 0;
        int qc = 4;
        // predecessor row / base for the three choices a record can make (m1, m4, d)
        int p1 = 0, b1 = 4, p4 = 0, b4 = 4, pd = 0;
        if (ri >= 0) {
            const RowDesc rd = load_desc(desc + ri);
            bsbe = rd.bsbe; d = rd.d;
            const int Bs = bsbe & 0xffff, Be = bsbe >> 16;
            const int j = cj - Bs * BLK;
            if (j >= 0 && j < (Be - Bs - 1) * BLK)
                rec = d >= 2 ? *reinterpret_cast<const uint32_t*>(tb + rd.tb + j * 4) : (uint32_t)tb[rd.tb + j];
            if (cj > 0) qc = qs[cj];
            p1 = p4 = pd = rd.prow0;
            b1 = b4 = rd.pbase;
            if (d >= 2) {
                const Rec r = decode_wide(rec);
                if (r.m1 >= 0) { p1 = in_row[rd.e0 + r.m1]; b1 = in_base[rd.e0 + r.m1]; }
                if (r.m4 >= 0) { p4 = in_row[rd.e0 + r.m4]; b4 = in_base[rd.e0 + r.m4]; }
                if (r.dpos >= 0) pd = in_row[rd.e0 + r.dpos];
            }
        }
        for (int t = 0; t < 32; t++) {
            const int Bs_t = __shfl_sync(0xffffffffu, bsbe, t) & 0xffff;
            const int Be_t = __shfl_sync(0xffffffffu, bsbe, t) >> 16;
            const int d_t = __shfl_sync(0xffffffffu, d, t);
            const uint32_t rec_t = __shfl_sync(0xffffffffu, rec, t);
            const int qc_t = __shfl_sync(0xffffffffu, qc, t);
            const int p1_t = __shfl_sync(0xffffffffu, p1, t), b1_t = __shfl_sync(0xffffffffu, b1, t);
            const int p4_t = __shfl_sync(0xffffffffu, p4, t), b4_t = __shfl_sync(0xffffffffu, b4, t);
            const int pd_t = __shfl_sync(0xffffffffu, pd, t);
            if (acj > (Be_t - 1) * BLK || acj < Bs_t * BLK) { status = ST_BAND_ESCAPE; break; }
            const int j = acj - Bs_t * BLK;
            if (j >= (Be_t - Bs_t - 1) * BLK) { status = ST_BT_FAIL; break; }
            if (nm + 1 > moves_cap) { status = ST_OOM; break; }
            const Rec r = d_t >= 2 ? decode_wide(rec_t) : decode_small((uint8_t)rec_t);
            int ni = i, na = acj;
            bool moved = false;
            if ((op & M_OP) && acj > 0 && r.m1 >= 0) {
                if (lane == 0) moves[nm] = mv_pack(b1_t == qc_t ? MV_MATCH : MV_MISMATCH, p1_t, qc_t);
                nm++;
                op = ALL_OP; ni = p1_t; na = acj - 1; moved = true;
            } else if ((op & D_OP) && (op == D_OP || r.eqMD) && r.dpos >= 0) {
                ni = pd_t;
                op = r.dext ? D_OP : (M_OP | I_OP);
                moved = true;
            } else if ((op & I_OP) && acj > 0 && j >= 1 && (op == I_OP || r.eqMI) && (r.iopen || r.iext)) {
                if (lane == 0) moves[nm] = mv_pack(MV_INSERT, 0, qc_t);
                nm++;
                op = r.iopen ? (M_OP | D_OP) : I_OP;
                na = acj - 1; moved = true;
            } else if ((op & M_OP) && acj > 0 && r.m4 >= 0) {
                if (lane == 0) moves[nm] = mv_pack(b4_t == qc_t ? MV_MATCH : MV_MISMATCH, p4_t, qc_t);
                nm++;
                op = ALL_OP; ni = p4_t; na = acj - 1; moved = true;
            }
            if (!moved) { status = ST_BT_FAIL; break; }
            i = ni;
            acj = na;
            if (!(i > 0 || acj > 0)) break;
            if (t + 1 >= 32 || i != i0 - (t + 1) || acj != a0 - (t + 1)) break;
        }
    }
    nm_out = nm;
    __syncwarp();
    return status;
}

// Build the DP rows of window [rank(source), rank(sink)] with the whole warp.
__device__ int build_view(DevGraph& g, char* s, const SlotLayout& L, WinView& v, int lane, bool recs) {
    const int beg_i = g.rank[0], end_i = g.rank[1];
    const int n = end_i - beg_i + 1;
    int32_t* in_ptr = (int32_t*)(s + L.v_in_ptr);
    int32_t* out_ptr = (int32_t*)(s + L.v_out_ptr);
    int32_t* in_row = (int32_t*)(s + L.v_in_row);
    int32_t* in_w = (int32_t*)(s + L.v_in_w);
    uint8_t* in_base = (uint8_t*)(s + L.v_in_base);
    int32_t* out_row = (int32_t*)(s + L.v_out_row);
    uint8_t* vb = (uint8_t*)(s + L.v_base);
    int32_t* vind = (int32_t*)(s + L.v_ind);
    int32_t* hq = (int32_t*)(s + L.v_hq);
    int32_t* hq_loc = (int32_t*)(s + L.v_hq_loc);
    int32_t* tq = (int32_t*)(s + L.v_tq);
    const int h0 = g.hlen[beg_i], t0 = g.tlen[end_i];
    // pass 1: per-row counts and scalars
    for (int r = lane; r < n; r += 32) {
        const int u = g.rank_to_id[beg_i + r];
        int ci = 0, co = 0;
        for (int e = g.in_head[u]; e >= 0; e = g.e_nin[e]) ci += (g.rank[g.e_from[e]] - beg_i >= 0);
        for (int e = g.out_head[u]; e >= 0; e = g.e_nout[e]) co += (g.rank[g.e_to[e]] - beg_i < n);
        in_ptr[r + 1] = ci;
        out_ptr[r + 1] = co;
        vb[r] = g.base[u];
        vind[r] = g.ind[u];
        hq[r] = g.hlen[beg_i + r] - h0;
        hq_loc[r] = g.hlen[r] - h0;
        tq[r] = g.tlen[beg_i + r] - t0;
    }
    __syncwarp();
    // exclusive scans of the counts
    int ci_carry = 0, co_carry = 0;
    if (lane == 0) { in_ptr[0] = 0; out_ptr[0] = 0; }
    for (int c0 = 0; c0 < n; c0 += 32) {
        const int r = c0 + lane;
        int ci = r < n ? in_ptr[r + 1] : 0, co = r < n ? out_ptr[r + 1] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int yi = __shfl_up_sync(0xffffffffu, ci, o), yo = __shfl_up_sync(0xffffffffu, co, o);
            if (lane >= o) { ci += yi; co += yo; }
        }
        __syncwarp();
        if (r < n) { in_ptr[r + 1] = ci + ci_carry; out_ptr[r + 1] = co + co_carry; }
        ci_carry += __shfl_sync(0xffffffffu, ci, 31);
        co_carry += __shfl_sync(0xffffffffu, co, 31);
    }
    __syncwarp();
    // pass 2: fill the lists in in-list / out-list order
    for (int r = lane; r < n; r += 32) {
        const int u = g.rank_to_id[beg_i + r];
        int k = in_ptr[r];
        for (int e = g.in_head[u]; e >= 0; e = g.e_nin[e]) {
            const int p = g.rank[g.e_from[e]] - beg_i;
            if (p < 0) continue;
            in_row[k] = p;
            in_w[k] = g.e_w[e];
            in_base[k] = p == 0 ? 4 : g.base[g.e_from[e]];
            k++;
        }
        k = out_ptr[r];
        for (int e = g.out_head[u]; e >= 0; e = g.e_nout[e]) {
            const int sr = g.rank[g.e_to[e]] - beg_i;
            if (sr >= n) continue;
            out_row[k++] = sr;
        }
    }
    __syncwarp();
    if (recs) {
        // for the warp fill: each row's predecessor records in the backtrack's
        // priority order (in_weight descending, in-list position ascending),
        // erec = {predecessor row, 0, in_weight | position << 16,
        //         base | (in_weight >= ind/10) << 8}; the fill patches in the
        // predecessor's band and row-store location when it reaches the row.
        // Also each row's furthest successor row (row-store placement).
        int4* erec = (int4*)(s + L.v_pmeta);
        int32_t* vmaxs = (int32_t*)(s + L.v_desc);
        for (int r = lane; r < n; r += 32) {
            const int e0 = in_ptr[r], d = r == 0 ? 0 : in_ptr[r + 1] - e0;
            const int ind = vind[r];
            for (int k = 0; k < d; k++) {
                const int w = in_w[e0 + k];
                const int4 rec = make_int4(in_row[e0 + k], 0, (w & 0xffff) | (k << 16),
                                           (int)in_base[e0 + k] | ((w >= ind / 10) ? 256 : 0));
                int at = k;
                while (at > 0) {
                    const int4 prev = erec[e0 + at - 1];
                    if ((prev.z & 0xffff) >= w) break;  // ties keep list order
                    erec[e0 + at] = prev;
                    at--;
                }
                erec[e0 + at] = rec;
            }
            int maxs = r;
            for (int k = out_ptr[r]; k < out_ptr[r + 1]; k++) maxs = max(maxs, out_row[k]);
            vmaxs[r] = maxs;
        }
        __syncwarp();
    }
    v.n = n;
    v.in_ptr = in_ptr; v.in_row = in_row; v.in_w = in_w; v.in_base = in_base;
    v.base = vb; v.ind = vind; v.hq = hq; v.hq_loc = hq_loc; v.tq = tq;
    v.out_ptr = out_ptr; v.out_row = out_row;
    return beg_i;
}

template <bool STATIC>
__device__ void process_window(const BatchArgs& A, char* s, DpArgs& a, unsigned char* wsm, int w, int lane) {
    const SlotLayout& L = A.L;
    DevGraph g = slot_graph(s, L);
    const int r0 = A.win_off[w], r1 = A.win_off[w + 1];
    const bool lens = A.f > 0;
    constexpr bool static_band = STATIC;  // f > 0 && !ab_band (checked on the host)
    int status = ST_OK;
    // the window's counters: in registers for the adaptive-band kernel; in the
    // window's output slots (lane 0) for the static-band kernel, whose fill
    // runs faster with the registers free (measured)
    int64_t cells_r = 0, ecells_r = 0;
    long long ph_r[NPHASE] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t* const cells_g = A.cells + 2 * (int64_t)w;
    int64_t* const ph_g = A.phase + (int64_t)w * NPHASE;
    if (STATIC && lane == 0) {
        cells_g[0] = cells_g[1] = 0;
        for (int k = 0; k < NPHASE; k++) ph_g[k] = 0;
    }
    long long tc = clock64();
    auto tick = [&](int k) {
        long long t = clock64();
        if constexpr (STATIC) {
            if (lane == 0) ph_g[k] += t - tc;
        } else {
            ph_r[k] += t - tc;
        }
        tc = t;
    };
    auto add_cells = [&](int64_t c, int64_t e) {  // lane 0
        if constexpr (STATIC) {
            cells_g[0] += c;
            cells_g[1] += e;
        } else {
            cells_r += c;
            ecells_r += e;
        }
    };
    for (int x = lane; x < L.NC; x += 32) { g.hlen[x] = 0; g.tlen[x] = 0; }
    if (lane == 0) {
        int nn = 0;
        dg_add_node(g, nn, 4);
        dg_add_node(g, nn, 4);
        g.hdr[0] = nn;
        g.hdr[1] = 0;
    }
    __syncwarp();
    for (int r = r0; r < r1 && status == ST_OK; r++) {
        const uint8_t* rd = A.seq + A.read_off[r];
        const int len = A.read_len[r];
        if (len > L.QC) { status = ST_CAPACITY; break; }
        const int nn0 = g.hdr[0];
        if (nn0 <= 2) {  // src/align.cpp:1747-1753: source + one new node per base
            if (lane == 0) {
                int nn = nn0, ne = g.hdr[1], anchored = 0, st = ST_OK;
                for (int j = 0; j < len && st == ST_OK; j++) {
                    const int cur = dg_add_node(g, nn, nt4_dev(rd[j]));
                    if (cur < 0 || !dg_add_adj(g, ne, anchored, cur)) st = ST_CAPACITY;
                    anchored = cur;
                }
                if (st == ST_OK && !dg_add_adj(g, ne, anchored, 1)) st = ST_CAPACITY;
                g.hdr[0] = nn;
                g.hdr[1] = ne;
                g.hdr[2] = st;
                A.rstats[(int64_t)r * NRSTAT + 3] = nn;
                A.rstats[(int64_t)r * NRSTAT + 6] = ne;
            }
            __syncwarp();
            status = g.hdr[2];
            tick(PH_FUSE);
            if (status == ST_OK && r + 1 < r1)
                dg_topsort_warp(g, g.hdr[0], g.hdr[1], lens, (uint16_t*)wsm, A.smem_per_warp, lane);
            tick(PH_SORT);
            continue;
        }
        tick(PH_FUSE);
        // DP rows of the whole graph and the shifted query
        WinView v;
        int beg_i;
        if constexpr (static_band) {
            const int st = build_view_static(g, s, L, v, len + 1, A.f, A.b + (len + 1) / A.f, A.sring_rows,
                                             A.sring_blocks, lane, beg_i);
            if (st != ST_OK) { status = st; break; }
        } else {
            beg_i = build_view(g, s, L, v, lane, true);
        }
        uint8_t* qs = (uint8_t*)(s + L.qs);
        const int64_t qsb = qs_bytes(len);
        for (int64_t x = lane; x < qsb; x += 32) qs[x] = (x >= 2 && x < len + 2) ? nt4_dev(rd[x - 2]) : 4;
        if (lane == 0) {
            a.v = v;
            a.qs = qs;
            a.qlen = len;
            a.ab_band = A.ab_band;
            a.f = A.f;
            a.w = A.b + (A.f ? (len + 1) / A.f : 0);
            a.sc = A.sc;
            a.meta = (RowMeta*)(s + L.meta);
            a.state = (int32_t*)(s + L.state);
            a.rs = (int32_t*)(s + L.rs);
            a.rs_cap = L.rs_cap;
            a.ring_rows = L.ring_rows;
            a.ring_blocks = L.ring_blocks;
            a.tb = (uint8_t*)(s + L.tb);
            a.tb_cap = L.tb_cap;
            a.moves = (int32_t*)(s + L.moves);
            a.moves_cap = L.NC + L.QC + 16;
            a.out = g.hdr + 4;
        }
        __syncwarp();
        if (v.n > L.NC) { status = ST_CAPACITY; break; }
        tick(PH_VIEW);
        if constexpr (static_band) {
            // the query goes after the row ring in this warp's shared memory
            uint8_t* qsm = wsm + (size_t)A.sring_rows * A.sring_blocks * 64;
            for (int64_t x = lane * 16; x < qsb; x += 32 * 16)
                *reinterpret_cast<uint4*>(qsm + x) = *reinterpret_cast<const uint4*>(qs + x);
            __syncwarp();
            unsigned char* stage = qsm + ((qsb + 15) & ~(int64_t)15);
            dp_fill_warp_static(a, (const RowDesc*)(s + L.v_desc), (const int4*)(s + L.v_pmeta), (int32_t*)wsm,
                                A.sring_blocks, qsm, stage, lane);
        } else {
            // shared memory: staged records, the update's inputs, and the query when it fits
            const uint8_t* qf = qs;
            int4* sed = reinterpret_cast<int4*>(wsm);
            const int64_t sed_bytes = (int64_t)DYN_STAGE_EDGES * 16;
            int32_t* upd = reinterpret_cast<int32_t*>(wsm + sed_bytes);
            if (sed_bytes + UPD_BYTES + qsb <= A.smem_per_warp) {
                uint8_t* qsm = wsm + sed_bytes + UPD_BYTES;
                for (int64_t x = lane * 16; x < qsb; x += 32 * 16)
                    *reinterpret_cast<uint4*>(qsm + x) = *reinterpret_cast<const uint4*>(qs + x);
                qf = qsm;
            }
            __syncwarp();
            dp_fill_warp_dyn(a, (int4*)(s + L.v_pmeta), (const int32_t*)(s + L.v_desc), qf, sed, upd, lane);
        }
        __syncwarp();
        {
            // per-read band statistics
            int mbn = 0;
            long long mid = 0;
            for (int i = lane; i < v.n; i += 32) {
                const RowMeta rm = ((const RowMeta*)(s + L.meta))[i];
                mbn = max(mbn, rm.Be - rm.Bs - 1);
                mid += (long long)(rm.Bs + rm.Be - 1) * (BLK / 2);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                mbn = max(mbn, __shfl_xor_sync(0xffffffffu, mbn, o));
                mid += __shfl_xor_sync(0xffffffffu, mid, o);
            }
            if (lane == 0) {
                int32_t* o = A.rstats + (int64_t)r * NRSTAT;
                o[0] = mbn;
                o[1] = a.out[3];
                o[2] = v.n;
                o[7] = v.n > 0 ? (int32_t)(mid * 1000 / ((long long)v.n * (len + 1))) : 0;
                o[4] = a.out[4];  // record bytes and spilled row-store entries
                o[5] = a.out[5];
            }
        }
        tick(PH_FILL);
        if constexpr (static_band) {
            int st = a.out[0];
            int32_t nm = 0;
            if (st == ST_OK)
                st = bt_warp_static((const RowDesc*)(s + L.v_desc), a.v.in_row, a.v.in_base, a.tb, qs, v.n, len + 1,
                                    a.moves, a.moves_cap, nm, lane);
            if (lane == 0) {
                add_cells(a.out[3], a.out[6]);
                g.hdr[2] = st;
                g.hdr[13] = nm;
                g.hdr[12] = g.hdr[12] + 1;  // fusion stamp, increasing over the slot's lifetime
            }
        } else if (lane == 0) {
            int st = a.out[0];
            add_cells(a.out[3], a.out[6]);
            int32_t nm = 0;
            if (st == ST_OK) st = backtrack_records(a, len + 1, nm);
            g.hdr[2] = st;
            g.hdr[13] = nm;
            g.hdr[12] = g.hdr[12] + 1;
        }
        __syncwarp();
        tick(PH_BT);
        {
            int st = g.hdr[2];
            const int nm = g.hdr[13];
            if (st == ST_OK) {
                st = dg_fuse_warp(g, a.moves, nm, beg_i, (int32_t*)(s + L.path), g.hdr[12], lane);
                if (st == -1) {
                    // sequential fusion (a path that repeats a node or an aligned sibling)
                    st = ST_OK;
                    if (lane == 0) st = dg_fuse_seq(g, a.moves, nm, beg_i);
                    __syncwarp();
                }
            }
            if (lane == 0) g.hdr[2] = st;
        }
        __syncwarp();
        status = g.hdr[2];
        if (lane == 0) {
            A.rstats[(int64_t)r * NRSTAT + 3] = g.hdr[0];
            A.rstats[(int64_t)r * NRSTAT + 6] = g.hdr[1];
        }
        tick(PH_FUSE);
        if (status == ST_OK && r + 1 < r1)
            dg_topsort_warp(g, g.hdr[0], g.hdr[1], lens, (uint16_t*)wsm, A.smem_per_warp, lane);
        tick(PH_SORT);
    }
    if (lane == 0) {
        int len = -1;
        if (status == ST_OK) {
            len = dg_consensus(g, g.hdr[0], A.cons + (int64_t)w * A.cons_stride, A.cons_stride);
            if (len < 0) status = ST_CAPACITY;
        }
        tick(PH_CONS);
        A.cons_len[w] = len < 0 ? 0 : len;
        A.status[w] = status;
        if constexpr (!STATIC) {
            cells_g[0] = cells_r;
            cells_g[1] = ecells_r;
            for (int k = 0; k < NPHASE; k++) ph_g[k] = ph_r[k];
        }
    }
    __syncwarp();
}

template <int WARPS, bool STATIC, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) k_batch(BatchArgs A) {
    __shared__ DpArgs s_args[WARPS];
    extern __shared__ __align__(16) unsigned char dsm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t slot = (int64_t)blockIdx.x * WARPS + warp;
    char* s = A.slots + slot * A.L.bytes;
    unsigned char* wsm = dsm + (size_t)warp * A.smem_per_warp;
    while (true) {
        int idx = 0;
        if (lane == 0) idx = atomicAdd(A.counter, 1);
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= A.n_windows) break;
        process_window<STATIC>(A, s, s_args[warp], wsm, A.order[idx], lane);
    }
}

}  // namespace

BatchEngine::BatchEngine(int device) : device_(device) {
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    cudaStream_t s;
    cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    stream_ = s;
    cudaEvent_t e[5];
    for (int i = 0; i < 5; i++) cuda_check(cudaEventCreate(&e[i]), "cudaEventCreate");
    ev0_ = e[0];
    ev1_ = e[1];
    evr0_ = e[2];
    evr1_ = e[3];
    evp_ = e[4];
}

BatchEngine::~BatchEngine() {
    cudaSetDevice(device_);
    if (d_in_) cudaFree(d_in_);
    if (d_out_) cudaFree(d_out_);
    if (d_slots_) cudaFree(d_slots_);
    if (h_out_) cudaFreeHost(h_out_);
    for (void* e : {ev0_, ev1_, evr0_, evr1_, evp_})
        if (e) cudaEventDestroy((cudaEvent_t)e);
    if (kgraph_exec_) cudaGraphExecDestroy((cudaGraphExec_t)kgraph_exec_);
    if (stream_) cudaStreamDestroy((cudaStream_t)stream_);
}

void BatchEngine::ensure(void** ptr, size_t* cap, size_t bytes) {
    if (bytes <= *cap) return;
    if (*ptr) cuda_check(cudaFree(*ptr), "cudaFree");
    *ptr = nullptr;
    *cap = 0;
    cuda_check(cudaMalloc(ptr, bytes), "cudaMalloc(batch)");
    *cap = bytes;
}

void BatchEngine::upload(const BatchInput& in, const Params& p) {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    if (p.enable_seeding || p.progressive || p.result != 0)
        throw std::invalid_argument("batched windows support the consensus mode without -S/-p");
    p_ = p;
    set_plan(nullptr, nullptr, nullptr, nullptr);
    n_windows_ = in.n_windows;
    n_reads_ = in.n_reads;
    max_len_ = 0;
    max_win_bases_ = 0;
    std::vector<int64_t> cost(n_windows_);
    for (int r = 0; r < n_reads_; r++) max_len_ = std::max(max_len_, in.read_len[r]);
    for (int w = 0; w < n_windows_; w++) {
        int64_t b = 0;
        for (int r = in.win_off[w]; r < in.win_off[w + 1]; r++) b += in.read_len[r];
        max_win_bases_ = std::max(max_win_bases_, b);
        cost[w] = b * (in.win_off[w + 1] - in.win_off[w] + 1);
    }
    order_.resize(n_windows_);
    std::iota(order_.begin(), order_.end(), 0);
    std::stable_sort(order_.begin(), order_.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    cons_stride_ = (int32_t)((2 * (int64_t)max_len_ + 64 + 15) / 16 * 16);

    off_seq_ = 0;
    size_t o = up256((size_t)in.seq_bytes + 16);
    off_roff_ = o; o = up256(o + 8 * (size_t)n_reads_);
    off_rlen_ = o; o = up256(o + 4 * (size_t)n_reads_);
    off_woff_ = o; o = up256(o + 4 * (size_t)(n_windows_ + 1));
    off_order_ = o; o = up256(o + 4 * (size_t)n_windows_);
    off_ctr_ = o; o = up256(o + 64);
    ensure(&d_in_, &d_in_cap_, o);
    cudaStream_t s = (cudaStream_t)stream_;
    char* d = (char*)d_in_;
    cuda_check(cudaMemcpyAsync(d + off_seq_, in.seq, (size_t)in.seq_bytes, cudaMemcpyHostToDevice, s), "H2D seq");
    cuda_check(cudaMemcpyAsync(d + off_roff_, in.read_off, 8 * (size_t)n_reads_, cudaMemcpyHostToDevice, s), "H2D");
    cuda_check(cudaMemcpyAsync(d + off_rlen_, in.read_len, 4 * (size_t)n_reads_, cudaMemcpyHostToDevice, s), "H2D");
    cuda_check(cudaMemcpyAsync(d + off_woff_, in.win_off, 4 * (size_t)(n_windows_ + 1), cudaMemcpyHostToDevice, s),
               "H2D");
    cuda_check(cudaMemcpyAsync(d + off_order_, order_.data(), 4 * (size_t)n_windows_, cudaMemcpyHostToDevice, s),
               "H2D");
    stats.h2d_bytes = (int64_t)(in.seq_bytes + 12 * (int64_t)n_reads_ + 8 * (int64_t)n_windows_);

    out_cons_ = 0;
    o = up256((size_t)n_windows_ * cons_stride_);
    out_len_ = o; o = up256(o + 4 * (size_t)n_windows_);
    out_status_ = o; o = up256(o + 4 * (size_t)n_windows_);
    out_cells_ = o; o = up256(o + 16 * (size_t)n_windows_);
    out_phase_ = o; o = up256(o + 8 * (size_t)NPHASE * n_windows_);
    out_rstats_ = o; o = up256(o + 4 * (size_t)NRSTAT * n_reads_);
    out_bytes_ = o;
    ensure(&d_out_, &d_out_cap_, o);
    if (h_out_cap_ < o) {
        if (h_out_) cuda_check(cudaFreeHost(h_out_), "cudaFreeHost");
        h_out_ = nullptr;
        cuda_check(cudaMallocHost(&h_out_, o), "cudaMallocHost");
        h_out_cap_ = o;
    }
    cuda_check(cudaStreamSynchronize(s), "upload");
}

void BatchEngine::run() {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    stats.kernel_ms = 0.0;
    stats.retried = 0;
    stats.launches = 0;
    stats.fallback = 0;
    stats.plan_ms = 0.0;
    cudaStream_t rs = (cudaStream_t)stream_;
    cuda_check(cudaEventRecord((cudaEvent_t)evr0_, rs), "event");
    if (proposer_) {
        std::vector<int32_t> nodes;
        std::vector<int64_t> tb, spill;
        std::vector<float> cost;
        proposer_->plan(device_windows(), PROP_K, PROP_W, nodes, tb, spill, cost);
        set_plan(nodes.data(), tb.data(), spill.data(), cost.data());
        cuda_check(cudaEventRecord((cudaEvent_t)evp_, rs), "event");
    }
    if (n_reads_ > 0)
        cuda_check(cudaMemsetAsync((char*)d_out_ + out_rstats_, 0, 4 * (size_t)NRSTAT * n_reads_, rs),
                   "memset read stats");
    // With a plan, one pass sized by the plan's largest window, in the plan's
    // cost order; its windows that outgrow their slot fall back to the sizing
    // below. Without one, a first pass with capacities estimated from the read
    // lengths. Windows that outgrow their slot (ST_CAPACITY / ST_OOM) are re-run
    // with doubled capacities, up to three times.
    int first = 1;
    if (!plan_nodes_.empty()) {
        Caps c;
        c.NC = 64;
        c.tb_cap = 4096;
        c.spill = 0;
        for (int w = 0; w < n_windows_; w++) {
            c.NC = std::max<int64_t>(c.NC, plan_nodes_[w]);
            c.tb_cap = std::max(c.tb_cap, plan_tb_[w]);
            c.spill = std::max(c.spill, plan_spill_[w]);
        }
        c.NC = std::min<int64_t>(c.NC, 60000);
        launch(plan_order_.data(), n_windows_, c, PLAN_HEADROOM);
        first = 0;
    } else {
        launch(order_.data(), n_windows_, default_caps(1));
    }
    for (int attempt = first ? 2 : 1; attempt <= 8; attempt *= 2) {
        cudaStream_t s = (cudaStream_t)stream_;
        char* h = (char*)h_out_;
        cuda_check(cudaMemcpyAsync(h + out_status_, (char*)d_out_ + out_status_, 4 * (size_t)n_windows_,
                                   cudaMemcpyDeviceToHost, s), "D2H status");
        cuda_check(cudaStreamSynchronize(s), "D2H status");
        const int32_t* st = (const int32_t*)(h + out_status_);
        std::vector<int32_t> redo;
        for (int w = 0; w < n_windows_; w++)
            if (st[w] == ST_CAPACITY || st[w] == ST_OOM) redo.push_back(w);
        if (redo.empty()) break;
        if (attempt == 1) stats.fallback = (int32_t)redo.size();
        else stats.retried += (int32_t)redo.size();
        launch(redo.data(), (int32_t)redo.size(), default_caps(attempt));
    }
    cuda_check(cudaEventRecord((cudaEvent_t)evr1_, rs), "event");
    cuda_check(cudaEventSynchronize((cudaEvent_t)evr1_), "batch run");
    float ms = 0.f;
    cuda_check(cudaEventElapsedTime(&ms, (cudaEvent_t)evr0_, (cudaEvent_t)evr1_), "elapsed");
    stats.run_ms = ms;
    if (proposer_) {
        cuda_check(cudaEventElapsedTime(&ms, (cudaEvent_t)evr0_, (cudaEvent_t)evp_), "elapsed");
        stats.plan_ms = ms;
    }
}

int BatchEngine::ring_blocks() const {
    const int m = max_len_ + 1;
    const int wb = p_.b + (p_.f ? m / p_.f : 0);
    // adaptive rows can grow to the full query width: their ring rows are full width
    int rb = p_.f > 0 && !p_.ab_band ? std::min(m / BLK + 2, (2 * wb) / BLK + 4) : m / BLK + 2;
    return std::max(rb, 4);
}

BatchEngine::Caps BatchEngine::default_caps(int scale) const {
    // capacities estimated from the read lengths, scaled on retries
    const bool adaptive = p_.f > 0 && p_.ab_band;
    const int m = max_len_ + 1;
    const int wb = p_.b + (p_.f ? m / p_.f : 0);
    const int64_t est = 2 + (int64_t)max_len_ + (int64_t)(0.2 * (double)max_win_bases_) + 256;
    const int64_t NC64 = std::min<int64_t>(std::min<int64_t>(2 + max_win_bases_, est * scale), 60000);
    Caps c;
    c.NC = (int32_t)std::max<int64_t>(NC64, 64);
    const int rb = ring_blocks();
    const int tb_blocks = adaptive ? std::min(m / BLK + 2, (std::min(m / BLK + 2, (4 * wb) / BLK + 4)) * scale) : rb;
    c.tb_cap = (int64_t)c.NC * tb_blocks * BLK * 2 * std::min(scale, 2) + 4096;
    const int64_t spill_rows = std::min<int64_t>(c.NC, std::max<int64_t>(c.NC / (adaptive ? 8 : 4), 64) * scale);
    c.spill = spill_rows * rb * 16;
    return c;
}

void BatchEngine::set_plan(const int32_t* nodes, const int64_t* tb_bytes, const int64_t* spill, const float* cost) {
    if (!nodes) {
        plan_nodes_.clear();
        plan_tb_.clear();
        plan_spill_.clear();
        plan_order_.clear();
        return;
    }
    plan_nodes_.assign(nodes, nodes + n_windows_);
    plan_tb_.assign(tb_bytes, tb_bytes + n_windows_);
    plan_spill_.assign(spill, spill + n_windows_);
    plan_order_.resize(n_windows_);
    std::iota(plan_order_.begin(), plan_order_.end(), 0);
    std::stable_sort(plan_order_.begin(), plan_order_.end(), [&](int a, int b) { return cost[a] > cost[b]; });
}

void BatchEngine::launch(const int32_t* windows, int32_t count, const Caps& caps, double headroom) {
    cudaStream_t s = (cudaStream_t)stream_;
    int sms = 0;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_), "attr");
    const bool adaptive = p_.f > 0 && p_.ab_band;
    const int32_t NC = std::max(caps.NC, 64);
    const int32_t EC = 3 * NC;
    const int32_t QC = max_len_ + 8;
    const int ring_blocks = this->ring_blocks();
    const int32_t ring_rows = 32;
    const int64_t tb_cap = (caps.tb_cap + 4095) / 4096 * 4096;
    const int64_t spill = (caps.spill + 63) / 64 * 64;
    SlotLayout L = make_layout(NC, EC, QC, ring_rows, ring_blocks, spill, tb_cap, adaptive);
    const SlotLayout L_planned = L;
    const int warps = warps_per_block;
    const int smem_w = smem_per_warp;
    const size_t dyn = (size_t)warps * smem_w;
    // static band: shared-memory ring of up to 8 rows of ring_blocks blocks
    int sring_blocks = ring_blocks;
    const int qsm_bytes = (int)((qs_bytes(QC) + 15) / 16 * 16);
    const int stage_bytes = STAGE_ROWS * (int)sizeof(RowDesc) + STAGE_EDGES * 16;
    int sring_rows = std::min(8, (smem_w - qsm_bytes - stage_bytes) / std::max(1, sring_blocks * 64));
    if (sring_rows < 2) sring_rows = 0;
    if (p_.f > 0 && !p_.ab_band && qsm_bytes + stage_bytes > smem_w)
        throw std::invalid_argument("reads too long for the batch kernel's shared memory; raise smem_per_warp");
    if (!(p_.f > 0 && !p_.ab_band) && smem_w < DYN_STAGE_EDGES * 16 + UPD_BYTES)
        throw std::invalid_argument("smem_per_warp too small for the adaptive-band fill");
    if (smem_w % 16 != 0) throw std::invalid_argument("smem_per_warp must be a multiple of 16");
    int occ = 0;
    auto occ_of = [&](auto kern) {
        cuda_check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn), "smem attr");
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, warps * 32, dyn), "occupancy");
    };
    const bool stat = p_.f > 0 && !p_.ab_band;
    if (warps != 4) throw std::invalid_argument("batch kernel is built for 4 warps per block");
    // two register budgets: 3 blocks (12 warps) per SM at up to 168 registers, or
    // 4 blocks (16 warps) per SM at up to 128 registers
    const bool dense = blocks_per_sm >= 4;
    if (stat) { if (dense) occ_of(k_batch<4, true, 4>); else occ_of(k_batch<4, true, 3>); }
    else { if (dense) occ_of(k_batch<4, false, 4>); else occ_of(k_batch<4, false, 3>); }
    // every block must be resident at once (persistent kernel): never more than the occupancy allows
    const int per_sm = std::max(1, std::min(blocks_per_sm, occ));
    int blocks = sms * per_sm;
    if (max_blocks > 0) blocks = std::min(blocks, max_blocks);
    // and the slots must fit the device-memory budget (75 % of what is free, counting our own slots)
    size_t free_b = 0, total_b = 0;
    cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const size_t budget = (size_t)(0.75 * (double)(free_b + d_slots_cap_));
    if (headroom > 1.0) {
        // planned capacities: grow every slot by up to `headroom` while every resident
        // warp still gets one, so a window a little beyond the plan still fits
        const int want = std::max(1, std::min(blocks, (count + warps - 1) / warps));
        const double fit = 0.97 * (double)budget / ((double)want * warps * (double)L_planned.bytes);
        const double h = std::min(headroom, fit);
        if (h > 1.0) {
            const int32_t NCh = (int32_t)std::min<double>(60000.0, std::max(64.0, NC * h));
            const int64_t tbh = ((int64_t)(tb_cap * h) + 4095) / 4096 * 4096;
            const int64_t sph = ((int64_t)(spill * h) + 63) / 64 * 64;
            L = make_layout(NCh, 3 * NCh, QC, ring_rows, ring_blocks, sph, tbh, adaptive);
        }
    }
    const int64_t max_by_mem = (int64_t)(budget / (size_t)L.bytes) / warps;
    if (max_by_mem < 1) throw std::runtime_error("not enough device memory for one batch slot");
    blocks = (int)std::min<int64_t>(blocks, max_by_mem);
    blocks = std::min(blocks, (count + warps - 1) / warps);
    blocks = std::max(blocks, 1);
    const int64_t slots = (int64_t)blocks * warps;
    const size_t slot_total = (size_t)(slots * L.bytes);
    if (slot_total > d_slots_cap_) {
        if (d_slots_) cuda_check(cudaFree(d_slots_), "cudaFree");
        d_slots_ = nullptr;
        d_slots_cap_ = 0;
        cuda_check(cudaMalloc(&d_slots_, slot_total), "cudaMalloc(batch slots)");
        d_slots_cap_ = slot_total;
        // zeroed once: fusion stamps and slot headers start from a known state
        cuda_check(cudaMemsetAsync(d_slots_, 0, d_slots_cap_, s), "memset slots");
    }
    stats.slots = (int32_t)slots;
    stats.slot_bytes = L.bytes;

    char* d = (char*)d_in_;
    char* o = (char*)d_out_;
    cuda_check(cudaMemcpyAsync(d + off_order_, windows, 4 * (size_t)count, cudaMemcpyHostToDevice, s), "H2D order");
    BatchArgs A;
    std::memset(&A, 0, sizeof A);  // padding too: the graph cache compares the bytes
    A.seq = (const uint8_t*)(d + off_seq_);
    A.read_off = (const int64_t*)(d + off_roff_);
    A.read_len = (const int32_t*)(d + off_rlen_);
    A.win_off = (const int32_t*)(d + off_woff_);
    A.order = (const int32_t*)(d + off_order_);
    A.counter = (int32_t*)(d + off_ctr_);
    A.n_windows = count;
    A.sc = scoring_of(p_);
    A.b = p_.b;
    A.f = p_.f;
    A.ab_band = p_.ab_band;
    A.slots = (char*)d_slots_;
    A.L = L;
    A.smem_per_warp = smem_w;
    A.sring_rows = sring_rows;
    A.sring_blocks = sring_blocks;
    A.cons = o + out_cons_;
    A.cons_stride = cons_stride_;
    A.cons_len = (int32_t*)(o + out_len_);
    A.status = (int32_t*)(o + out_status_);
    A.cells = (int64_t*)(o + out_cells_);
    A.phase = (int64_t*)(o + out_phase_);
    A.rstats = (int32_t*)(o + out_rstats_);
    // the work-counter reset and the persistent launch, recorded as a CUDA graph and
    // replayed while the launch (variant, grid, shared memory, arguments) is unchanged
    struct KKey {
        bool stat, dense;
        int blocks;
        size_t dyn;
        BatchArgs A;
    } key;
    std::memset(&key, 0, sizeof key);
    key.stat = stat;
    key.dense = dense;
    key.blocks = blocks;
    key.dyn = dyn;
    key.A = A;
    if (!kgraph_exec_ || kgraph_key_.size() != sizeof key || std::memcmp(kgraph_key_.data(), &key, sizeof key) != 0) {
        if (kgraph_exec_) cudaGraphExecDestroy((cudaGraphExec_t)kgraph_exec_);
        kgraph_exec_ = nullptr;
        cudaGraph_t gr = nullptr;
        cuda_check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
        cudaMemsetAsync(A.counter, 0, 4, s);
        if (stat) {
            if (dense) k_batch<4, true, 4><<<blocks, 4 * 32, dyn, s>>>(A);
            else k_batch<4, true, 3><<<blocks, 4 * 32, dyn, s>>>(A);
        } else {
            if (dense) k_batch<4, false, 4><<<blocks, 4 * 32, dyn, s>>>(A);
            else k_batch<4, false, 3><<<blocks, 4 * 32, dyn, s>>>(A);
        }
        const cudaError_t le = cudaGetLastError();
        const cudaError_t ce = cudaStreamEndCapture(s, &gr);
        cuda_check(le, "k_batch launch");
        cuda_check(ce, "end capture");
        cudaGraphExec_t ex = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&ex, gr, 0);
        cudaGraphDestroy(gr);
        cuda_check(ie, "graph instantiate");
        kgraph_exec_ = ex;
        kgraph_key_.assign((const char*)&key, (const char*)&key + sizeof key);
    }
    cuda_check(cudaEventRecord((cudaEvent_t)ev0_, s), "event");
    cuda_check(cudaGraphLaunch((cudaGraphExec_t)kgraph_exec_, s), "k_batch graph launch");
    cuda_check(cudaEventRecord((cudaEvent_t)ev1_, s), "event");
    cuda_check(cudaEventSynchronize((cudaEvent_t)ev1_), "k_batch");
    float ms = 0.f;
    cuda_check(cudaEventElapsedTime(&ms, (cudaEvent_t)ev0_, (cudaEvent_t)ev1_), "elapsed");
    stats.kernel_ms += ms;
    stats.launches++;
}

void BatchEngine::sync_stats() {
    cudaStream_t s = (cudaStream_t)stream_;
    char* h = (char*)h_out_;
    const size_t a = out_status_, b = out_bytes_;
    cuda_check(cudaMemcpyAsync(h + a, (char*)d_out_ + a, b - a, cudaMemcpyDeviceToHost, s), "D2H stats");
    cuda_check(cudaStreamSynchronize(s), "D2H stats");
    const int32_t* st = (const int32_t*)(h + out_status_);
    const int64_t* cl = (const int64_t*)(h + out_cells_);
    const int64_t* ph = (const int64_t*)(h + out_phase_);
    stats.cells = 0;
    stats.edge_cells = 0;
    stats.failed = 0;
    for (int k = 0; k < 8; k++) stats.phase_cycles[k] = 0;
    for (int w = 0; w < n_windows_; w++) {
        stats.cells += cl[2 * (int64_t)w];
        stats.edge_cells += cl[2 * (int64_t)w + 1];
        stats.failed += st[w] != ST_OK;
        for (int k = 0; k < NPHASE; k++) stats.phase_cycles[k] += ph[(int64_t)w * NPHASE + k];
    }
}

void BatchEngine::download(std::vector<std::string>& cons, std::vector<int32_t>& status) {
    cudaStream_t s = (cudaStream_t)stream_;
    char* h = (char*)h_out_;
    cuda_check(cudaMemcpyAsync(h, d_out_, out_bytes_, cudaMemcpyDeviceToHost, s), "D2H out");
    cuda_check(cudaStreamSynchronize(s), "D2H out");
    stats.d2h_bytes = (int64_t)out_bytes_;
    const int32_t* ln = (const int32_t*)(h + out_len_);
    const int32_t* st = (const int32_t*)(h + out_status_);
    const int64_t* cl = (const int64_t*)(h + out_cells_);
    cons.resize(n_windows_);
    status.resize(n_windows_);
    stats.cells = 0;
    stats.edge_cells = 0;
    stats.failed = 0;
    for (int w = 0; w < n_windows_; w++) {
        cons[w].assign(h + out_cons_ + (size_t)w * cons_stride_, (size_t)ln[w]);
        status[w] = st[w];
        stats.cells += cl[2 * (int64_t)w];
        stats.edge_cells += cl[2 * (int64_t)w + 1];
        stats.failed += st[w] != ST_OK;
    }
}

}  // namespace pb

namespace pb {

DeviceWindows BatchEngine::device_windows() const {
    DeviceWindows d;
    const char* b = (const char*)d_in_;
    d.seq = (const uint8_t*)(b + off_seq_);
    d.read_off = (const int64_t*)(b + off_roff_);
    d.read_len = (const int32_t*)(b + off_rlen_);
    d.win_off = (const int32_t*)(b + off_woff_);
    d.n_reads = n_reads_;
    d.n_windows = n_windows_;
    d.max_len = max_len_;
    d.max_win_bases = max_win_bases_;
    d.stream = stream_;
    return d;
}

void BatchEngine::read_stats(std::vector<int32_t>& out) {
    cudaStream_t s = (cudaStream_t)stream_;
    out.resize((size_t)NRSTAT * n_reads_);
    if (n_reads_ == 0) return;
    cuda_check(cudaMemcpyAsync(out.data(), (char*)d_out_ + out_rstats_, 4 * (size_t)NRSTAT * n_reads_,
                               cudaMemcpyDeviceToHost, s), "D2H read stats");
    cuda_check(cudaStreamSynchronize(s), "D2H read stats");
}

}  // namespace pb
