/*
 * poa_oracle.c - scalar CPU restatement of minipoa's POA hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels, never shipped or
 * measured as the product. Every function cites the reference lines it
 * restates. The restatement is deliberately naive (one cell at a time, full
 * int32 M/D/I rows kept for the backtrack) so that it is easy to audit
 * against the reference; speed is not a goal.
 *
 * One intentional deviation: the reference never initialises the I row of the
 * window's first rank (src/align.cpp:1412-1424 writes only M and D) yet its
 * backtrack may read it at (row 0, column > 0). Such a read needs a path
 * whose score is NEG_INF-derived, since M[0][j>0] = NEG_INF. The restatement
 * defines that row as NEG_INF.
 */
#include "poa_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ utils */
typedef struct { int *a; int n, cap; } ivec;

static void iv_push(ivec *v, int x) {
    if (v->n == v->cap) {
        v->cap = v->cap ? v->cap * 2 : 4;
        v->a = (int *)realloc(v->a, (size_t)v->cap * sizeof(int));
    }
    v->a[v->n++] = x;
}
static void iv_free(ivec *v) { free(v->a); v->a = NULL; v->n = v->cap = 0; }
static void iv_resize_keep(ivec *v, int n) { /* std::vector::resize: keep, zero-fill new */
    while (v->cap < n) {
        v->cap = v->cap ? v->cap * 2 : 16;
        v->a = (int *)realloc(v->a, (size_t)v->cap * sizeof(int));
    }
    for (int i = v->n; i < n; i++) v->a[i] = 0;
    v->n = n;
}

static inline int32_t add32(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
static inline int32_t max32(int32_t a, int32_t b) { return a > b ? a : b; }
static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* src/sequence.cpp:6-23: A/C/G/T (either case) -> 0..3, bytes 0..3 map to
 * themselves (so double encoding is harmless), everything else -> 4. */
uint8_t po_nt4(uint8_t c) {
    switch (c) {
    case 0: case 1: case 2: case 3: return c;
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': case 'U': case 'u': return 3;
    default: return 4;
    }
}
static const char po_nt256[5] = {'A', 'C', 'G', 'T', 'N'}; /* src/sequence.cpp:26-43 */

/* ------------------------------------------------------------------ params */
void po_params_default(po_params *p) { /* src/main.cpp:18-33 */
    p->match = 2; p->mismatch = -4; p->gap_open1 = -4; p->gap_ext1 = -2;
    p->b = 100; p->f = 40; p->ab_band = 0; p->verbose = 0;
}
void po_params_normalize(po_params *p) { /* src/handle_input.cpp:47-50 */
    /* :47 negates para->m (not match) when match < 0; match keeps its sign */
    if (p->mismatch > 0) p->mismatch = -p->mismatch;
    if (p->gap_open1 > 0) p->gap_open1 = -p->gap_open1;
    if (p->gap_ext1 > 0) p->gap_ext1 = -p->gap_ext1;
}

/* ------------------------------------------------------------------ graph */
typedef struct {
    int id, rank, par_id, ind;
    uint8_t base;
    int aligned[5];
    ivec in, in_w, out, out_w, ids, idp;
} po_node;

struct po_graph {
    po_node *node; int n, cap;
    ivec rank;        /* rank -> node id */
    ivec hlen, tlen;  /* indexed by rank; std::vector resize semantics */
    int is_topsorted;
};

static int g_new_node(po_graph *g, uint8_t base) { /* node_t ctor, include/node.h:16-22 */
    if (g->n == g->cap) {
        g->cap = g->cap ? g->cap * 2 : 64;
        g->node = (po_node *)realloc(g->node, (size_t)g->cap * sizeof(po_node));
    }
    po_node *v = &g->node[g->n];
    memset(v, 0, sizeof(*v));
    v->id = v->par_id = g->n;
    v->base = base;
    v->rank = 0;
    for (int k = 0; k < 5; k++) v->aligned[k] = -1;
    v->aligned[base] = v->id;
    return g->n++;
}

po_graph *po_graph_new(void) { /* graph::init, src/graph.cpp:129-135 */
    po_graph *g = (po_graph *)calloc(1, sizeof(po_graph));
    g_new_node(g, 4); /* source 0 */
    g_new_node(g, 4); /* sink 1   */
    return g;
}
void po_graph_free(po_graph *g) {
    if (!g) return;
    for (int i = 0; i < g->n; i++) {
        po_node *v = &g->node[i];
        iv_free(&v->in); iv_free(&v->in_w); iv_free(&v->out); iv_free(&v->out_w);
        iv_free(&v->ids); iv_free(&v->idp);
    }
    free(g->node); iv_free(&g->rank); iv_free(&g->hlen); iv_free(&g->tlen);
    free(g);
}
int po_graph_nnodes(const po_graph *g) { return g->n; }
const int *po_graph_rank_to_id(const po_graph *g, int *n) { *n = g->rank.n; return g->rank.a; }
int po_graph_node_base(const po_graph *g, int id) { return g->node[id].base; }

/* node_t::add_in_adj / add_out_adj, include/node.h:23-61; graph::add_adj, src/graph.cpp:13-20 */
static void g_add_adj(po_graph *g, int seq_id, int from, int to, int cur_pos) {
    if (from == to) return;
    po_node *f = &g->node[from];
    int ok = 0;
    for (int i = 0; i < f->out.n; i++)
        if (f->out.a[i] == to) { f->out_w.a[i]++; ok = 1; break; }
    if (!ok) { iv_push(&f->out, to); iv_push(&f->out_w, 1); }
    if (f->ids.n == 0 || f->ids.a[f->ids.n - 1] != seq_id) iv_push(&f->ids, seq_id);

    po_node *t = &g->node[to];
    t->ind++;
    ok = 0;
    for (int i = 0; i < t->in.n; i++)
        if (t->in.a[i] == from) { t->in_w.a[i]++; ok = 1; break; }
    if (!ok) { iv_push(&t->in, from); iv_push(&t->in_w, 1); }
    if (t->ids.n == 0 || t->ids.a[t->ids.n - 1] != seq_id) {
        iv_push(&t->ids, seq_id);
        iv_push(&t->idp, cur_pos);
    }
}

/* graph::add_path, src/graph.cpp:170-235 */
void po_add_path(po_graph *g, int seq_id, const po_res *res, int n, int sink_id) {
    int anchored = -1, cur_pos = 0;
    for (int i = 0; i < n; i++) {
        int cur = res[i].from;
        if (cur < 0) {
            if (res[i].aligned_id >= 0) {
                int al = res[i].aligned_id;
                if (g->node[al].aligned[res[i].base] == -1) {
                    cur = g_new_node(g, res[i].base);
                    g->node[al].aligned[res[i].base] = cur;
                    g->node[cur].par_id = al;
                } else {
                    cur = g->node[al].aligned[res[i].base];
                }
            } else {
                cur = g_new_node(g, res[i].base);
            }
        }
        if (anchored != -1) g_add_adj(g, seq_id, anchored, cur, cur_pos++);
        anchored = cur;
    }
    if (sink_id != -1) g_add_adj(g, seq_id, anchored, sink_id, cur_pos);
    g->is_topsorted = 0;
}

/* graph::topsort, src/graph.cpp:21-128 (op 0: LIFO Kahn + hlen/tlen;
 * op 1: one rank per aligned-node group, the MSA columns). */
void po_topsort(po_graph *g, const po_params *p, int op) {
    int N = g->n;
    int *deg = (int *)calloc((size_t)N, sizeof(int));
    int *stk = (int *)malloc((size_t)(N + 1) * sizeof(int));
    int sp = 0;
    g->rank.n = 0;
    if (op == 1) {
        for (int i = 0; i < N; i++) {
            po_node *v = &g->node[i];
            v->rank = -1;
            if (v->par_id != v->id) continue;
            int s = 0;
            for (int k = 0; k < 5; k++)
                if (v->aligned[k] >= 0) s += g->node[v->aligned[k]].in.n;
            deg[i] = s;
            if (s == 0) stk[sp++] = i;
        }
        while (sp) {
            int u = stk[--sp];
            po_node *cur = &g->node[u];
            cur->rank = g->rank.n;
            iv_push(&g->rank, u);
            for (int k = 0; k < 5; k++) {
                if (cur->aligned[k] < 0) continue;
                po_node *son = &g->node[cur->aligned[k]];
                son->rank = cur->rank;
                for (int j = 0; j < son->out.n; j++) {
                    int v = g->node[son->out.a[j]].par_id;
                    if (--deg[v] == 0) stk[sp++] = v;
                }
            }
        }
        g->is_topsorted = 1;
        free(deg); free(stk);
        return;
    }
    for (int i = 0; i < N; i++) {
        deg[i] = g->node[i].in.n;
        if (deg[i] == 0) stk[sp++] = i;
    }
    while (sp) {
        int u = stk[--sp];
        po_node *cur = &g->node[u];
        cur->rank = g->rank.n;
        iv_push(&g->rank, u);
        for (int k = 0; k < cur->out.n; k++) {
            int v = cur->out.a[k];
            if (--deg[v] == 0) stk[sp++] = v;
        }
    }
    g->is_topsorted = 1;
    if (p->f > 0) {
        iv_resize_keep(&g->hlen, N);
        for (int i = 0; i < g->rank.n; i++) {
            po_node *cur = &g->node[g->rank.a[i]];
            int wmax = -1, max_pre = -1;
            for (int k = 0; k < cur->in.n; k++)
                if (cur->in_w.a[k] > wmax) { wmax = cur->in_w.a[k]; max_pre = g->node[cur->in.a[k]].rank; }
            if (max_pre != -1) g->hlen.a[cur->rank] = g->hlen.a[max_pre] + 1;
        }
        iv_resize_keep(&g->tlen, N);
        g->tlen.a[g->node[1].rank] = 1;
        for (int i = g->rank.n - 1; i >= 0; i--) {
            po_node *cur = &g->node[g->rank.a[i]];
            int wmax = -1, max_suc = -1;
            for (int k = 0; k < cur->out.n; k++)
                if (cur->out_w.a[k] > wmax) { wmax = cur->out_w.a[k]; max_suc = g->node[cur->out.a[k]].rank; }
            if (max_suc != -1) g->tlen.a[cur->rank] = g->tlen.a[max_suc] + 1;
        }
    }
    free(deg); free(stk);
}

/* graph::build_consensus, src/graph.cpp:294-351 (FIFO Kahn from the source,
 * heaviest in-edge, ties to the larger accumulated score, first wins). */
static int *g_consensus_ids(const po_graph *g, int *len) {
    int N = g->n;
    int *deg = (int *)calloc((size_t)N, sizeof(int));
    int *pre = (int *)calloc((size_t)N, sizeof(int));
    int *score = (int *)calloc((size_t)N, sizeof(int));
    int *q = (int *)malloc((size_t)(N + 1) * sizeof(int));
    int qh = 0, qt = 0;
    for (int i = 0; i < N; i++) deg[i] = g->node[i].in.n;
    q[qt++] = 0;
    while (qh < qt) {
        int u = q[qh++];
        const po_node *cur = &g->node[u];
        if (u != 0) {
            int wmax = -1, max_pre = -1;
            for (int k = 0; k < cur->in.n; k++) {
                int pr = g->node[cur->in.a[k]].id;
                int wk = cur->in_w.a[k];
                if (wk > wmax || (wk == wmax && score[pr] > score[max_pre])) { wmax = wk; max_pre = pr; }
            }
            pre[u] = max_pre;
            score[u] = score[max_pre] + wmax;
        }
        if (u == 1) break;
        for (int k = 0; k < cur->out.n; k++) {
            int v = cur->out.a[k];
            if (--deg[v] == 0) q[qt++] = v;
        }
    }
    int n = 0;
    for (int id = pre[1]; id != 0; id = pre[id]) n++;
    int *ids = (int *)malloc((size_t)(n + 1) * sizeof(int));
    int k = n;
    for (int id = pre[1]; id != 0; id = pre[id]) ids[--k] = id;
    *len = n;
    free(deg); free(pre); free(score); free(q);
    return ids;
}

char *po_consensus(const po_graph *g, int *len) {
    int n;
    int *ids = g_consensus_ids(g, &n);
    char *s = (char *)malloc((size_t)n + 1);
    for (int i = 0; i < n; i++) s[i] = po_nt256[g->node[ids[i]].base];
    s[n] = 0;
    free(ids);
    *len = n;
    return s;
}

/* graph::output_rc_msa, src/graph.cpp:237-251 (after the op==1 topsort). */
char *po_msa(const po_graph *g, int nseq, int *ncol) {
    int nc = g->rank.n - 2;
    if (nc < 0) nc = 0;
    char *rows = (char *)malloc((size_t)nseq * (size_t)nc + 1);
    memset(rows, '-', (size_t)nseq * (size_t)nc);
    for (int i = 2; i < g->n; i++) {
        const po_node *v = &g->node[i];
        int rk = g->node[v->par_id].rank;
        if (rk - 1 < 0 || rk - 1 >= nc) continue; /* out of range in the reference too */
        for (int t = 0; t < v->ids.n; t++) {
            int id = v->ids.a[t];
            if (id >= 0 && id < nseq) rows[(size_t)id * nc + (rk - 1)] = po_nt256[v->base];
        }
    }
    rows[(size_t)nseq * nc] = 0;
    *ncol = nc;
    return rows;
}

/* ------------------------------------------------------------------ GFA */
typedef struct { char *a; size_t n, cap; } sbuf;
static void sb_put(sbuf *b, const char *s) {
    size_t k = strlen(s);
    if (b->n + k + 1 > b->cap) {
        b->cap = (b->n + k + 1) * 2;
        b->a = (char *)realloc(b->a, b->cap);
    }
    memcpy(b->a + b->n, s, k + 1);
    b->n += k;
}

/* graph::output_gfa, src/graph.cpp:358-434: H line; S and L lines in FIFO
 * Kahn order from the source, stopping at the sink (L lines per in-edge in
 * in-list order, source edges left out); read paths from each node's
 * (read ord, position) pairs. A P line has no "\t*\n" when its read is empty
 * (the reference writes the terminator only after the last position). */
char *po_gfa(const po_graph *g, int nseq, const int *lens, const char *const *names) {
    sbuf b = {0, 0, 0};
    sb_put(&b, "");
    if (g->n <= 2) return b.a;
    int *deg = (int *)malloc(sizeof(int) * (size_t)g->n);
    int *queue = (int *)malloc(sizeof(int) * (size_t)g->n);
    int **paths = (int **)calloc((size_t)(nseq > 0 ? nseq : 1), sizeof(int *));
    for (int i = 0; i < g->n; i++) deg[i] = g->node[i].in.n;
    for (int i = 0; i < nseq; i++) paths[i] = (int *)calloc((size_t)(lens[i] > 0 ? lens[i] : 1), sizeof(int));
    char line[128];
    sb_put(&b, "H\tVN:Z:1.0\n");
    int head = 0, tail = 0;
    queue[tail++] = 0;
    while (head < tail) {
        const int cur = queue[head++];
        if (cur == 1) break;
        const po_node *v = &g->node[cur];
        if (cur != 0) {
            snprintf(line, sizeof line, "S\t%d\t%c\n", cur - 1, po_nt256[v->base]);
            sb_put(&b, line);
            for (int k = 0; k < v->in.n; k++) {
                const int pre = v->in.a[k];
                if (pre == 0) continue;
                snprintf(line, sizeof line, "L\t%d\t+\t%d\t+\t0M\n", pre - 1, cur - 1);
                sb_put(&b, line);
            }
            for (int k = 0; k < v->ids.n && k < v->idp.n; k++) {
                const int id = v->ids.a[k], pos = v->idp.a[k];
                if (id >= 0 && id < nseq && pos >= 0 && pos < lens[id]) paths[id][pos] = cur - 1;
            }
        }
        for (int k = 0; k < v->out.n; k++) {
            const int o = v->out.a[k];
            if (--deg[o] == 0) queue[tail++] = o;
        }
    }
    for (int i = 0; i < nseq; i++) {
        if (names && names[i] && names[i][0]) {
            sb_put(&b, "P\t");
            sb_put(&b, names[i]);
            sb_put(&b, "\t");
        } else {
            snprintf(line, sizeof line, "P\t%d\t", i + 1);
            sb_put(&b, line);
        }
        for (int j = 0; j < lens[i]; j++) {
            snprintf(line, sizeof line, "%d+%s", paths[i][j], j + 1 < lens[i] ? "," : "\t*\n");
            sb_put(&b, line);
        }
    }
    for (int i = 0; i < nseq; i++) free(paths[i]);
    free(paths);
    free(queue);
    free(deg);
    return b.a;
}

/* ------------------------------------------------------------------ poa() */
enum { M_OP = 1, D_OP = 2, I_OP = 4, ALL_OP = 7 };

typedef struct { po_res *a; int n, cap; } rvec;
static void rv_push(rvec *v, int from, uint8_t base, int aligned_id) {
    if (v->n == v->cap) {
        v->cap = v->cap ? v->cap * 2 : 64;
        v->a = (po_res *)realloc(v->a, (size_t)v->cap * sizeof(po_res));
    }
    v->a[v->n].from = from; v->a[v->n].base = base; v->a[v->n].aligned_id = aligned_id;
    v->n++;
}

/* poa(), src/align.cpp:1353-1737. */
int po_poa(const po_graph *g, const po_params *p, int beg_id, int end_id,
           const uint8_t *qin, int qlen, int ab_band, po_res **path, int *plen, int *score) {
    const po_node *node = g->node;
    const int *rank = g->rank.a;
    const int *hlen = g->hlen.a, *tlen = g->tlen.a;
    int beg_i = node[beg_id].rank, end_i = node[end_id].rank;
    int n = end_i - beg_i + 1, m = qlen + 1;
    if (n <= 0 || qlen < 0 || p->b < 0 || p->f < 0) return PO_BAD_ARG;
    const int match = p->match, mismatch = p->mismatch, e1 = p->gap_ext1, o1 = p->gap_open1 + p->gap_ext1;

    /* :1361-1366, :1371-1372: leading 'N' sentinel, 'N' padding to col_size */
    int col_size = (m + 1 + PO_BLK - 1) / PO_BLK * PO_BLK;
    uint8_t *seq = (uint8_t *)malloc((size_t)col_size);
    seq[0] = 4;
    for (int j = 0; j < qlen; j++) seq[j + 1] = po_nt4(qin[j]);
    for (int j = m; j < col_size; j++) seq[j] = 4;

    int *Ms = (int *)malloc(sizeof(int) * n), *Me = (int *)malloc(sizeof(int) * n);
    int *Bs = (int *)malloc(sizeof(int) * n), *Be = (int *)malloc(sizeof(int) * n);
    int *Mp = (int *)calloc(n, sizeof(int)), *Sl = (int *)calloc(n, sizeof(int));
    int *Pl = (int *)malloc(sizeof(int) * n), *Pr = (int *)calloc(n, sizeof(int));
    int *Ol = (int *)calloc(n, sizeof(int)), *Or = (int *)calloc(n, sizeof(int));
    int *Ow = (int *)calloc(n, sizeof(int));
    int32_t **M = (int32_t **)calloc(n, sizeof(int32_t *));
    int32_t **D = (int32_t **)calloc(n, sizeof(int32_t *));
    int32_t **I = (int32_t **)calloc(n, sizeof(int32_t *));
    for (int i = 0; i < n; i++) Pl[i] = m;

    int w = p->b;
    if (p->f) w += m / p->f;                             /* :1378-1379 */
    const int adaptive = (p->f > 0 && ab_band);
    for (int i = 0; i < n; i++) {                        /* :1382-1394 */
        int aci = beg_i + i;
        if (p->f > 0 && !ab_band) {
            int h = hlen[aci] - hlen[beg_i], t = m - tlen[aci] + tlen[end_i];
            Ms[i] = imax(0, imin(h, t) - w);
            Me[i] = imin(m, imax(h, t) + w);
        } else { Ms[i] = 0; Me[i] = m; }
        Bs[i] = Ms[i] / PO_BLK; Be[i] = Me[i] / PO_BLK + 2;
    }
    if (adaptive) {                                      /* :1410-1414 */
        int h = hlen[beg_i] - hlen[beg_i], t = m - tlen[beg_i] + tlen[end_i];
        Ms[0] = imax(0, imin(imin(Pl[0], h + Ol[0]), t) - w);
        Me[0] = imin(m, imax(imax(Pr[0], h + Or[0]), t) + w);
        Bs[0] = Ms[0] / PO_BLK; Be[0] = Me[0] / PO_BLK + 2;
    }
    { /* row 0, :1415-1423 */
        int width = (Be[0] - Bs[0]) * PO_BLK;
        M[0] = (int32_t *)malloc(sizeof(int32_t) * width);
        D[0] = (int32_t *)malloc(sizeof(int32_t) * width);
        I[0] = (int32_t *)malloc(sizeof(int32_t) * width);
        for (int j = 0; j < width; j++) { M[0][j] = PO_NEG_INF; D[0][j] = PO_NEG_INF; I[0][j] = PO_NEG_INF; }
        M[0][0] = 0;
    }
    for (int i = 1; i < n; i++) {                        /* :1426-1569 */
        int aci = beg_i + i;
        const po_node *cur = &node[rank[aci]];
        if (adaptive) {                                  /* :1433-1444 */
            int h = hlen[aci] - hlen[beg_i], t = m - tlen[aci] + tlen[end_i];
            Ms[i] = imax(0, imin(imin(Pl[i], h + Ol[i]), t) - w - Ow[i]);
            Me[i] = imin(m, imax(imax(Pr[i], h + Or[i]), t) + w + Ow[i]);
            Bs[i] = Ms[i] / PO_BLK; Be[i] = Me[i] / PO_BLK + 2;
        }
        int block_num = Be[i] - Bs[i] - 1;
        int width = (Be[i] - Bs[i]) * PO_BLK;
        int32_t *Mi = M[i] = (int32_t *)malloc(sizeof(int32_t) * width);
        int32_t *Di = D[i] = (int32_t *)malloc(sizeof(int32_t) * width);
        int32_t *Ii = I[i] = (int32_t *)malloc(sizeof(int32_t) * width);
        int pre_num = 0;
        for (int k = 0; k < cur->in.n; k++) {            /* :1449-1498 */
            const po_node *pre = &node[cur->in.a[k]];
            int pr = pre->rank - beg_i;
            if (pr < 0) continue;
            int pbase = pr == 0 ? 4 : pre->base;
            const int32_t *Mp_ = M[pr], *Dp_ = D[pr];
            for (int bid = 0; bid < block_num; bid++) {
                int acBid = Bs[i] + bid;
                int diag = !((imax(0, acBid - 1) < Bs[pr]) || (acBid > Be[pr] - 2));   /* :1467 */
                int vert = (Bs[pr] <= acBid && acBid < Be[pr] - 1);                    /* :1484 */
                for (int l = 0; l < PO_BLK; l++) {
                    int j = bid * PO_BLK + l, acj = acBid * PO_BLK + l;
                    int32_t Mij = pre_num == 0 ? PO_NEG_INF : Mi[j];
                    int32_t Dij = pre_num == 0 ? PO_NEG_INF : Di[j];
                    int pj = acj - Bs[pr] * PO_BLK;
                    if (diag) {
                        int qc = acj == 0 ? 4 : seq[acj - 1];
                        /* lane 0 of the row's first block reads NEG_INF (:1454, :1477) */
                        int32_t dv = (bid == 0 && l == 0) ? PO_NEG_INF : Mp_[pj - 1];
                        Mij = max32(Mij, add32(dv, pbase == qc ? match : mismatch));
                    }
                    if (vert) {
                        Dij = max32(Dij, add32(Dp_[pj], e1));
                        Dij = max32(Dij, add32(Mp_[pj], o1));
                    }
                    Mi[j] = Mij; Di[j] = Dij;
                }
            }
            pre_num++;
        }
        if (pre_num == 0)
            for (int j = 0; j < block_num * PO_BLK; j++) { Mi[j] = PO_NEG_INF; Di[j] = PO_NEG_INF; }
        for (int j = block_num * PO_BLK; j < width; j++) { Mi[j] = PO_NEG_INF; Di[j] = PO_NEG_INF; Ii[j] = PO_NEG_INF; }
        Ii[0] = PO_NEG_INF;                              /* :1507-1514 */
        Mi[0] = max32(max32(Mi[0], Di[0]), Ii[0]);
        for (int j = 1; j < block_num * PO_BLK; j++) {
            Ii[j] = max32(add32(Ii[j - 1], e1), add32(Mi[j - 1], o1));
            Mi[j] = max32(max32(Mi[j], Di[j]), Ii[j]);
        }
        if (adaptive) {                                  /* :1516-1568 */
            int max_j = 0;
            for (int j = 1; j < block_num * PO_BLK; j++) max_j = Mi[j] > Mi[max_j] ? j : max_j;
            int max_acj = Bs[i] * PO_BLK + max_j, max_slp = 0, is_match = 0;
            Mp[i] = max_acj;
            if (cur->base == seq[max_acj]) {
                for (int k = 0; k < cur->in.n; k++) {
                    int pr = node[cur->in.a[k]].rank - beg_i;
                    if (pr < 0) continue;
                    max_slp = Sl[pr] > max_slp ? Sl[pr] : max_slp;
                    if (Mp[pr] + 1 == Mp[i]) { Sl[i] = imax(Sl[i], Sl[pr] + 1); is_match = 1; }
                }
            }
            if (!is_match && max_slp < 30) {
                Ow[i] += max_slp + 1;
                Ow[i] = imin(Ow[i], 5 * w);
            }
            if (Sl[i] >= 30) {
                /* :1542-1543 index hlen by the window-local row i (as written) */
                Ol[i] = max_acj - (hlen[i] - hlen[beg_i]);
                Or[i] = max_acj - (hlen[i] - hlen[beg_i]);
                Ow[i] = 0;
                for (int k = 0; k < cur->out.n; k++) {
                    int s = node[cur->out.a[k]].rank - beg_i;
                    if (s >= n) continue;
                    Ol[s] = Ol[i]; Or[s] = Or[i];
                }
            }
            for (int k = 0; k < cur->out.n; k++) {
                int s = node[cur->out.a[k]].rank - beg_i;
                if (s >= n) continue;
                Ol[s] = imin(Ol[s], Ol[i]); Or[s] = imax(Or[s], Or[i]);
            }
            for (int k = 0; k < cur->out.n; k++) {
                int s = node[cur->out.a[k]].rank - beg_i;
                if (s >= n) continue;
                Pl[s] = imin(Pl[s], max_acj); Pr[s] = imax(Pr[s], max_acj + 1);
                Ow[s] = Ow[i] ? imax(Ow[s], Ow[i]) : Ow[i];
            }
        }
    }

    /* backtrack, :1572-1736 */
    int status = PO_OK;
    rvec res = {0};
    int i = n - 1, acj = m;
    *score = M[i][acj - Bs[i] * PO_BLK];
    int op = ALL_OP;
    while (i > 0 || acj > 0) {
        int j = acj - Bs[i] * PO_BLK;
        int aci = beg_i + i;
        if (acj > (Be[i] - 1) * PO_BLK || acj < Bs[i] * PO_BLK) { status = PO_BAND_ESCAPE; break; }
        const po_node *cur = &node[rank[aci]];
        const int32_t Mij = M[i][j];
        if ((op & M_OP) && acj > 0) {                    /* :1589-1624 */
            int bk = -1;
            for (int k = 0; k < cur->in.n; k++) {
                const po_node *pre = &node[cur->in.a[k]];
                int pr = pre->rank - beg_i;
                if (pr < 0) continue;
                int pbase = pr == 0 ? 4 : pre->base;
                if (pbase != seq[acj - 1]) continue;
                int pj = acj - Bs[pr] * PO_BLK;
                int bn = Be[pr] - Bs[pr] - 1;
                if (pj - 1 >= 0 && pj - 1 < bn * PO_BLK &&
                    Mij == add32(M[pr][pj - 1], pbase == seq[acj - 1] ? match : mismatch) &&
                    (bk == -1 || cur->in_w.a[k] > cur->in_w.a[bk]))
                    bk = k;
            }
            if (bk != -1 && cur->in_w.a[bk] >= cur->ind / 10) {
                const po_node *pre = &node[cur->in.a[bk]];
                int pr = pre->rank - beg_i;
                int pbase = pr == 0 ? 4 : pre->base;
                uint8_t qc = seq[acj - 1];
                if (pbase == qc) rv_push(&res, pre->id, pre->base, -1);
                else {
                    const po_node *par = &node[pre->par_id];
                    if (par->aligned[qc] != -1) rv_push(&res, par->aligned[qc], qc, -1);
                    else rv_push(&res, -1, qc, pre->par_id);
                }
                op = ALL_OP; i = pr; acj--;
                continue;
            }
        }
        if (op & D_OP) {                                 /* :1625-1665 */
            if (op == D_OP || Mij == D[i][j]) {
                int bk = -1, bop = 0;
                for (int k = 0; k < cur->in.n; k++) {
                    int pr = node[cur->in.a[k]].rank - beg_i;
                    if (pr < 0) continue;
                    if (Bs[pr] <= acj / PO_BLK && acj / PO_BLK < Be[pr] - 1) {
                        int pj = acj - Bs[pr] * PO_BLK;
                        if (D[i][j] == add32(M[pr][pj], o1) && (bk == -1 || cur->in_w.a[k] > cur->in_w.a[bk])) {
                            bk = k; bop = M_OP | I_OP;
                        }
                    }
                }
                if (bk == -1) {
                    for (int k = 0; k < cur->in.n; k++) {
                        int pr = node[cur->in.a[k]].rank - beg_i;
                        if (pr < 0) continue;
                        if (Bs[pr] <= acj / PO_BLK && acj / PO_BLK < Be[pr] - 1) {
                            int pj = acj - Bs[pr] * PO_BLK;
                            if (D[i][j] == add32(D[pr][pj], e1) && (bk == -1 || cur->in_w.a[k] > cur->in_w.a[bk])) {
                                bk = k; bop = D_OP;
                            }
                        }
                    }
                }
                if (bk != -1) {
                    i = node[cur->in.a[bk]].rank - beg_i;
                    op = bop;
                    continue;
                }
            }
        }
        if ((op & I_OP) && acj > 0) {                    /* :1666-1686 */
            if (j - 1 >= 0 && (op == I_OP || Mij == I[i][j])) {
                if (I[i][j] == add32(M[i][j - 1], o1)) {
                    rv_push(&res, -1, seq[acj - 1], -1);
                    op = M_OP | D_OP; acj--;
                    continue;
                }
                if (I[i][j] == add32(I[i][j - 1], e1)) {
                    rv_push(&res, -1, seq[acj - 1], -1);
                    op = I_OP; acj--;
                    continue;
                }
            }
        }
        if ((op & M_OP) && acj > 0) {                    /* :1687-1729 */
            int bk = -1;
            for (int k = 0; k < cur->in.n; k++) {
                const po_node *pre = &node[cur->in.a[k]];
                int pr = pre->rank - beg_i;
                if (pr < 0) continue;
                int pbase = pr == 0 ? 4 : pre->base;
                int pj = acj - Bs[pr] * PO_BLK;
                int bn = Be[pr] - Bs[pr] - 1;
                if (pj - 1 >= 0 && pj - 1 < bn * PO_BLK &&
                    Mij == add32(M[pr][pj - 1], pbase == seq[acj - 1] ? match : mismatch) &&
                    (bk == -1 || cur->in_w.a[k] > cur->in_w.a[bk]))
                    bk = k;
            }
            if (bk != -1) {
                op = ALL_OP;
                const po_node *pre = &node[cur->in.a[bk]];
                int pr = pre->rank - beg_i;
                int pbase = pr == 0 ? 4 : pre->base;
                uint8_t qc = seq[acj - 1];
                if (pbase == qc) rv_push(&res, pre->id, pre->base, -1);
                else {
                    const po_node *par = &node[pre->par_id];
                    if (par->aligned[qc] != -1) rv_push(&res, par->aligned[qc], qc, -1);
                    else rv_push(&res, -1, qc, pre->par_id);
                }
                i = pr; acj--;
                continue;
            }
        }
        status = PO_BT_FAIL;
        break;
    }
    for (int r = 0; r < n; r++) { free(M[r]); free(D[r]); free(I[r]); }
    free(M); free(D); free(I);
    free(Ms); free(Me); free(Bs); free(Be); free(Mp); free(Sl); free(Pl); free(Pr);
    free(Ol); free(Or); free(Ow); free(seq);
    if (status != PO_OK) { free(res.a); *path = NULL; *plen = 0; return status; }
    for (int a = 0, b = res.n - 1; a < b; a++, b--) { po_res t = res.a[a]; res.a[a] = res.a[b]; res.a[b] = t; }
    *path = res.a; *plen = res.n;
    return PO_OK;
}

/* alignment() without seeding, src/align.cpp:1741-1756 */
int po_alignment(const po_graph *g, const po_params *p, const uint8_t *q, int qlen,
                 po_res **path, int *plen, int *score) {
    if (g->n <= 2) {
        po_res *r = (po_res *)malloc(sizeof(po_res) * (size_t)(qlen + 1));
        r[0].from = 0; r[0].base = 4; r[0].aligned_id = -1;
        for (int j = 0; j < qlen; j++) { r[j + 1].from = -1; r[j + 1].base = po_nt4(q[j]); r[j + 1].aligned_id = -1; }
        *path = r; *plen = qlen + 1; *score = 0;
        return PO_OK;
    }
    return po_poa(g, p, 0, 1, q, qlen, p->ab_band, path, plen, score);
}

/* The driver loop, src/main.cpp:84-126 with the identity read order. */
char *po_run(const po_params *p, int nseq, const char *const *seqs, const int *lens,
             const char *const *names, int mode, int *scores, int *status) {
    (void)names;
    po_graph *g = po_graph_new();
    *status = PO_OK;
    for (int i = 0; i < nseq; i++) {
        po_res *path; int plen, sc;
        uint8_t *q = (uint8_t *)malloc((size_t)lens[i] + 1);
        for (int j = 0; j < lens[i]; j++) q[j] = po_nt4((uint8_t)seqs[i][j]);
        int st = po_alignment(g, p, q, lens[i], &path, &plen, &sc);
        free(q);
        if (st != PO_OK) { *status = st; po_graph_free(g); return NULL; }
        if (scores) scores[i] = sc;
        po_add_path(g, i, path, plen, 1);
        free(path);
        po_topsort(g, p, i + 1 == nseq);
    }
    char *out;
    if (mode == 0) {
        int len;
        char *c = po_consensus(g, &len);
        out = (char *)malloc((size_t)len + 32);
        sprintf(out, ">consensus sequence\n%s\n", c);
        free(c);
    } else {
        int nc;
        char *rows = po_msa(g, nseq, &nc);
        out = (char *)malloc((size_t)nseq * (size_t)(nc + 1) + 1);
        char *o = out;
        for (int i = 0; i < nseq; i++) {
            memcpy(o, rows + (size_t)i * nc, (size_t)nc); o += nc; *o++ = '\n';
        }
        *o = 0;
        free(rows);
    }
    po_graph_free(g);
    return out;
}

/* ------------------------------------------------------------------ export */
void po_graph_sizes(const po_graph *g, int *n_nodes, int *n_in, int *n_out, int *n_ranks, int *n_lens) {
    int ni = 0, no = 0;
    for (int i = 0; i < g->n; i++) { ni += g->node[i].in.n; no += g->node[i].out.n; }
    *n_nodes = g->n; *n_in = ni; *n_out = no; *n_ranks = g->rank.n; *n_lens = g->hlen.n;
}

void po_graph_export(const po_graph *g, uint8_t *base, int *rank, int *par, int *ind, int *aligned,
                     int *in_ptr, int *in_id, int *in_w, int *out_ptr, int *out_id, int *rank_to_id,
                     int *hlen, int *tlen) {
    int ki = 0, ko = 0;
    in_ptr[0] = out_ptr[0] = 0;
    for (int i = 0; i < g->n; i++) {
        const po_node *v = &g->node[i];
        base[i] = v->base; rank[i] = v->rank; par[i] = v->par_id; ind[i] = v->ind;
        for (int k = 0; k < 5; k++) aligned[5 * i + k] = v->aligned[k];
        for (int k = 0; k < v->in.n; k++) { in_id[ki] = v->in.a[k]; in_w[ki] = v->in_w.a[k]; ki++; }
        for (int k = 0; k < v->out.n; k++) out_id[ko++] = v->out.a[k];
        in_ptr[i + 1] = ki; out_ptr[i + 1] = ko;
    }
    for (int r = 0; r < g->rank.n; r++) rank_to_id[r] = g->rank.a[r];
    for (int r = 0; r < g->hlen.n; r++) hlen[r] = g->hlen.a[r];
    for (int r = 0; r < g->tlen.n; r++) tlen[r] = g->tlen.a[r];
}
