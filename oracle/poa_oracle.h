/*
 * poa_oracle.h - CPU restatement of minipoa's hot path (TEST INFRASTRUCTURE).
 *
 * This is the checker for the CUDA path, never the product: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg use it. It restates,
 * in plain scalar C, minipoa's banded affine-gap graph DP and backtrack
 * (src/align.cpp:1353-1737), the per-read dispatch without seeding
 * (src/align.cpp:1741-1756), graph fusion (src/graph.cpp:7-20, 170-235;
 * include/node.h:16-61), topological sort with hlen/tlen
 * (src/graph.cpp:21-128), consensus (src/graph.cpp:294-357) and the
 * row-column MSA (src/graph.cpp:237-251) and the GFA output
 * (src/graph.cpp:358-434).
 *
 * Parity is pinned against the reference itself: tests/golden/ holds outputs
 * of the unmodified reference (built by oracle/Makefile into oracle/_ref/) on
 * seeded inputs, per-call scores and paths from oracle/ref_harness.cpp, and
 * the restatement must reproduce every one of them byte for byte.
 */
#ifndef POA_ORACLE_H
#define POA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PO_NEG_INF ((int32_t)0xc0c0c0c0) /* src/align.cpp:22 */
#define PO_BLK 8                          /* AVX2 int32 lanes, src/align.cpp:13-19 */

/* Status codes (the reference exits instead, src/align.cpp:1584-1588,1730-1731). */
enum { PO_OK = 0, PO_BAND_ESCAPE = 1, PO_BT_FAIL = 2, PO_BAD_ARG = 3 };

typedef struct {
    int match, mismatch, gap_open1, gap_ext1; /* normalised like initPara */
    int b, f;                                 /* band: w = b + m/f        */
    int ab_band;                              /* -B                       */
    int verbose;
} po_params;

typedef struct { int from; uint8_t base; int aligned_id; } po_res; /* include/result.h:3-12 */

typedef struct po_graph po_graph;

void po_params_default(po_params *p);           /* src/main.cpp:16-33 defaults */
void po_params_normalize(po_params *p);         /* src/handle_input.cpp:45-51   */
uint8_t po_nt4(uint8_t ascii);                  /* src/sequence.cpp:6-23        */

po_graph *po_graph_new(void);                   /* graph::init, src/graph.cpp:129-147 */
void po_graph_free(po_graph *g);
int po_graph_nnodes(const po_graph *g);

/* One banded DP + backtrack over ranks [rank(beg_id), rank(end_id)].
 * q: encoded query (0..4), qlen bases. On PO_OK *path (malloc'd, caller frees)
 * holds *plen elements in forward order and *score the end-cell score. */
int po_poa(const po_graph *g, const po_params *p, int beg_id, int end_id,
           const uint8_t *q, int qlen, int ab_band, po_res **path, int *plen, int *score);

/* alignment() without seeding (src/align.cpp:1741-1756). *score is 0 when the
 * graph is empty (no DP). */
int po_alignment(const po_graph *g, const po_params *p, const uint8_t *q, int qlen,
                 po_res **path, int *plen, int *score);

void po_add_path(po_graph *g, int seq_id, const po_res *res, int n, int sink_id);
void po_topsort(po_graph *g, const po_params *p, int op);

/* Heaviest-path consensus; returns ASCII (malloc'd, NUL-terminated). */
char *po_consensus(const po_graph *g, int *len);
/* Row-column MSA: nseq rows of *ncol chars, row r for ord r (malloc'd block). */
char *po_msa(const po_graph *g, int nseq, int *ncol);
/* GFA text (-r 2, src/graph.cpp:358-434); lens/names per read in input order
 * (names may be NULL: reads are then numbered from 1). malloc'd. */
char *po_gfa(const po_graph *g, int nseq, const int *lens, const char *const *names);

/* Whole driver loop (src/main.cpp:84-126, default read order, no seeding).
 * seqs: ASCII. mode 0 = consensus, 1 = MSA. Returns malloc'd text exactly as
 * the reference prints it to stdout, or NULL on error (*status set).
 * If scores != NULL it receives one score per read (0 for the first). */
char *po_run(const po_params *p, int nseq, const char *const *seqs, const int *lens,
             const char *const *names, int mode, int *scores, int *status);

/* Flatten the graph for tests: sizes first (nodes, in-edges, out-edges,
 * ranks, hlen entries), then the arrays (caller-allocated; aligned has
 * 5 entries per node; in/out lists in list order as CSR). */
void po_graph_sizes(const po_graph *g, int *n_nodes, int *n_in, int *n_out, int *n_ranks, int *n_lens);
void po_graph_export(const po_graph *g, uint8_t *base, int *rank, int *par, int *ind, int *aligned,
                     int *in_ptr, int *in_id, int *in_w, int *out_ptr, int *out_id, int *rank_to_id,
                     int *hlen, int *tlen);

/* Per-graph introspection used by tests (arrays valid until the next mutation). */
const int *po_graph_rank_to_id(const po_graph *g, int *n);
int po_graph_node_base(const po_graph *g, int id);

#ifdef __cplusplus
}
#endif
#endif
