/*
 * poa_b200.h - C ABI of the B200 partial-order-alignment engine.
 *
 * Plain pointers and sizes only. Every entry point returns a status code
 * (POA_OK = 0) instead of exiting the process the way the reference does;
 * poa_status_str() names it and poa_last_error() gives the last message of a
 * context. Sequences are ASCII (A/C/G/T/N, either case) unless a parameter
 * says "encoded" (codes 0..4 = A, C, G, T, N, as src/sequence.cpp:6-23).
 *
 * The entry points replace these reference interfaces (paths within the
 * minipoa project):
 *   poa_params / poa_params_init  para_t and its CLI defaults,
 *                                 include/parameter.h:5-19, src/main.cpp:16-33,
 *                                 normalised like initPara, src/handle_input.cpp:45-51
 *   poa_align                     poa(), include/align.h:15, src/align.cpp:1353-1737
 *   poa_run                       the driver loop + output, src/main.cpp:84-126
 *                                 (alignment(), src/align.cpp:1741-1828; add_path,
 *                                 topsort, output_consensus / output_rc_msa /
 *                                 output_gfa,
 *                                 src/graph.cpp)
 *   poa_batch_*                   the same driver over many independent windows
 *                                 (no counterpart: the reference handles one
 *                                 graph per process)
 */
#ifndef POA_B200_H
#define POA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    POA_OK = 0,
    POA_BAND_ESCAPE = 1, /* reference: prints the band and exit(0), src/align.cpp:1584-1588 */
    POA_BT_FAIL = 2,     /* reference: " backtrack error" + exit(1), src/align.cpp:1730-1731 */
    POA_BAD_ARG = 3,
    POA_OOM = 4,         /* device memory exhausted */
    POA_INDEGREE = 5,    /* a node with more than 510 in-window predecessors */
    POA_DEGENERATE = 6,  /* an empty band / sub-window the reference cannot handle either */
    POA_CAPACITY = 7,    /* a batched window outgrew its device graph capacity */
    POA_CUDA = 8,        /* a CUDA runtime error; see poa_last_error() */
    POA_UNSUPPORTED = 9
};

/* para_t, the fields on the path. Values are the raw CLI values; signs are
 * normalised inside (initPara). */
typedef struct {
    int32_t match, mismatch, gap_open, gap_ext; /* -M -X -O -E: 2 -4 -4 -2 */
    int32_t band_b, band_f;                     /* -b -f: 100 40 */
    int32_t ab_band;                            /* -B: 0 */
    int32_t seeding;                            /* -S: 0 */
    int32_t k, mm_w, poa_w;                     /* -k -w -W: 19 10 0 (-W is read only when given) */
    int32_t thread;                             /* -t: 1 */
    int32_t result;                             /* -r: 0 consensus, 1 row-column MSA, 2 GFA */
    int32_t progressive;                        /* -p: 0 */
    int32_t verbose;                            /* -V: 0 */
} poa_params;

typedef struct poa_ctx poa_ctx;

void poa_params_init(poa_params* p);
const char* poa_status_str(int status);

/* One context per GPU and host thread; owns a CUDA stream and device memory. */
poa_ctx* poa_create(int device, const poa_params* p);
void poa_destroy(poa_ctx* ctx);
const char* poa_last_error(const poa_ctx* ctx);
void poa_free(void* ptr);

/* The reference graph flattened (node_t, include/node.h:5-68; graph,
 * include/graph.h:9-31). Arrays are indexed by node id unless stated. */
typedef struct {
    int32_t n_nodes;
    const uint8_t* base;     /* encoded base */
    const int32_t* rank;     /* node rank from the last topsort(op 0) */
    const int32_t* par_id;
    const int32_t* ind;      /* in-degree count incl. repeated edges */
    const int32_t* aligned;  /* [n_nodes * 5] aligned_node */
    const int32_t* in_ptr;   /* [n_nodes + 1] CSR in in-list order */
    const int32_t* in_id;
    const int32_t* in_weight;
    const int32_t* out_ptr;  /* [n_nodes + 1] CSR in out-list order */
    const int32_t* out_id;
    int32_t n_ranks;
    const int32_t* rank_to_id;
    const int32_t* hlen;     /* by rank; may be NULL when band_f == 0 */
    const int32_t* tlen;
} poa_graph_view;

/* res_t, include/result.h:3-12 */
typedef struct {
    int32_t from;
    uint8_t base;
    int32_t aligned_id;
} poa_res;

/* poa(): align the encoded query (qlen bases, codes 0..4) to ranks
 * [rank(beg_id), rank(end_id)] of the graph; writes the forward path to out
 * (capacity out_cap), its length to *out_len and the end-cell score to *score. */
int poa_align(poa_ctx* ctx, const poa_graph_view* g, int32_t beg_id, int32_t end_id, const uint8_t* q_enc,
              int32_t qlen, int32_t ab_band, poa_res* out, int32_t out_cap, int32_t* out_len, int32_t* score);

/* The whole minipoa run: reads in order, DP on the GPU, graph fusion on the
 * host, output text exactly as minipoa prints it (consensus FASTA for
 * result 0, one row per read for result 1, GFA for result 2, nothing for
 * other values). headers[i] is the text after '>' of read i ("name
 * comment"; GFA path lines use the name), or NULL / "" for ">i+1". *text is allocated
 * with malloc; release it with poa_free. scores (optional, nseq entries) gets
 * the end-cell score of each read's last poa() call (0 for the first read). */
int poa_run(poa_ctx* ctx, int32_t nseq, const char* const* seqs, const int32_t* lens,
            const char* const* headers, char** text, size_t* text_len, int32_t* scores);
/* poa_run on top of an existing graph, minipoa -i (read_gfa,
 * src/handle_input.cpp:444-494; src/main.cpp:86-126): gfa holds the GFA
 * text (S lines become nodes, P lines reads without bases; L/W lines are
 * ignored); the reads then extend that graph. The outputs list the GFA's
 * paths first, as the reference does. A malformed GFA returns POA_BAD_ARG
 * with the reason in poa_last_error. */
int poa_run_gfa(poa_ctx* ctx, const char* gfa, size_t gfa_len, int32_t nseq, const char* const* seqs,
                const int32_t* lens, const char* const* headers, char** text, size_t* text_len, int32_t* scores);

/* Batched windows (consensus mode, no -S/-p): many independent read sets,
 * one POA graph and one consensus each, all in one persistent launch on the
 * device; no counterpart in the reference, which handles one graph per
 * process (each window equals one minipoa run on its reads).
 * Reads are ASCII, read r = seq[read_off[r] .. read_off[r] + read_len[r]);
 * window w owns reads win_off[w] .. win_off[w+1]-1, aligned in that order.
 * poa_batch_upload copies them into device memory (kept resident),
 * poa_batch_run runs every window and returns the device time in ms, and
 * poa_batch_download writes window w's consensus to
 * cons[cons_off[w] .. cons_off[w+1]) (cons_cap bytes available; cons_off has
 * n_windows + 1 entries) and its status. poa_batch_consensus does all three. */
int poa_batch_upload(poa_ctx* ctx, const uint8_t* seq, int64_t seq_bytes, const int64_t* read_off,
                     const int32_t* read_len, int32_t n_reads, const int32_t* win_off, int32_t n_windows);
int poa_batch_run(poa_ctx* ctx, double* device_ms);
int poa_batch_download(poa_ctx* ctx, char* cons, int64_t cons_cap, int64_t* cons_off, int32_t* status);
int poa_batch_consensus(poa_ctx* ctx, const uint8_t* seq, int64_t seq_bytes, const int64_t* read_off,
                        const int32_t* read_len, int32_t n_reads, const int32_t* win_off, int32_t n_windows,
                        char* cons, int64_t cons_cap, int64_t* cons_off, int32_t* status);
/* The same from files, streamed (no counterpart in the reference beyond its
 * reader, src/handle_input.cpp:13-43): window w is the FASTA / FASTQ file
 * paths[w] (plain or gzip), read as one minipoa run reads its input. Files
 * go in chunks of `chunk` windows; `threads` host threads (0 = all cores)
 * read and parse chunk k+1 into page-locked memory while chunk k runs on the
 * device. A chunk should hold several times the resident windows (the
 * batch's slot count) to keep the device busy. Outputs as poa_batch_consensus for all
 * n_files windows; a file that cannot be read returns POA_BAD_ARG. */
int poa_batch_consensus_files(poa_ctx* ctx, const char* const* paths, int32_t n_files, int32_t chunk,
                              int32_t threads, char* cons, int64_t cons_cap, int64_t* cons_off, int32_t* status);
/* [0] band cells of the last run, [1] windows that failed, [2] concurrent
 * slots, [3] bytes per slot, [4] H2D bytes of the upload, [5] D2H bytes,
 * [6..11] summed per-window clock cycles of the view build, DP fill,
 * backtrack, graph fusion, topological sort and consensus phases,
 * [12] kernel launches of the last run, [13] windows re-run with larger
 * capacities, [14] windows that outgrew the plan's sizing (poa_batch_plan)
 * and were re-run with the default sizing, [15] device time of the batch
 * kernel launches of the last run in microseconds, [16] device time of the
 * whole last run (plan, launches, re-runs) in microseconds, [17] device time
 * of the proposer's plan in microseconds (0 without a proposer), [18] edge
 * cells of the last run (band cells x in-window predecessors of their row). */
int poa_batch_stats(poa_ctx* ctx, int64_t* out19);
/* Resource plan for the uploaded windows (no counterpart in the reference:
 * the reference allocates per alignment). One value per window: graph nodes,
 * traceback record bytes and spilled row-store entries (int32) of its
 * largest alignment, and a relative cost; typically a band proposer's
 * prediction from poa_batch_read_stats-style targets. The plan sizes the
 * device slots and orders the windows (largest cost first); it never changes
 * a band, so results are the same with or without it. A window that
 * outgrows its slot is re-run with the default sizing. nodes == NULL clears
 * the plan; poa_batch_upload clears it too. */
int poa_batch_plan(poa_ctx* ctx, const int32_t* nodes, const int64_t* tb_bytes, const int64_t* spill,
                   const float* cost);
/* The per-window plan the last run used (set by poa_batch_plan or the
 * proposer): graph nodes, record bytes of the largest alignment and spilled
 * row-store entries, n_windows values each. With poa_batch_read_stats it
 * shows how often a window's real need exceeded its own prediction, apart
 * from the slot headroom that the launch adds. */
int poa_batch_plan_get(poa_ctx* ctx, int32_t* nodes, int64_t* tb_bytes, int64_t* spill, int32_t n_windows);
/* Per read of the last run, 8 values each (n_reads * 8 entries): widest DP
 * row in 8-column blocks, band cells, DP rows, graph nodes after fusing the
 * read, traceback record bytes, spilled row-store entries (int32), graph
 * edges after fusing the read, 0. A window's first read has no DP: its DP
 * values are zero. These are the band statistics the band proposer learns. */
int poa_batch_read_stats(poa_ctx* ctx, int32_t* out, int64_t cap);

/* One poa() alignment on inputs already in device memory, without
 * allocating anything (no counterpart in the reference).
 *
 * For callers that cannot allocate at the time they align: code inside a
 * framework that owns the device memory pool, or a latency-bound service
 * that forbids cudaMalloc on its request path (cudaMalloc synchronises the
 * device and can fail under memory pressure). All arrays below are device
 * pointers the caller owns; the DP's working memory is a fixed array of
 * POA_NOALLOC_SCRATCH_BYTES inside the library, present on every GPU that
 * loads the library until the process exits.
 *
 * Limit: the window must fit that array at its worst case (every row at the
 * full band width): about n_rows * (96 * ((qlen + 1) / 8 + 1) + 68) bytes,
 * plus the query, must stay under POA_NOALLOC_SCRATCH_BYTES (64 MiB). That
 * is up to about 7,800 rows with a 700 bp query, or about 550 rows with a
 * 10 kb query. Larger windows are rejected with POA_OOM before anything is
 * launched; impossible sizes (negative, or a query whose buffer alone
 * exceeds the array) are rejected the same way, with no arithmetic that can
 * wrap. On a failed alignment result_dev[1..3] are 0.
 *
 * w: the window's rows (ranks beg..end), laid out like the rows poa_align
 * builds: CSR predecessor lists in in-list order (predecessor row, its
 * in_weight, its base with 'N' for row 0), node base and in-degree count per
 * row, hq = hlen[rank]-hlen[beg], hq_loc = hlen[row]-hlen[beg],
 * tq = tlen[rank]-tlen[end], CSR successor rows in out-list order.
 * q_dev: encoded query (codes 0..4). moves_dev (capacity moves_cap >=
 * n_rows + qlen + 1) receives the backtrack moves in backtrack order, each
 * (pred_row << 5 | kind << 3 | base) with kind 0 match, 1 mismatch,
 * 2 insertion; result_dev[4] receives status, score, number of moves and
 * band cells. The call is asynchronous on `stream` (a cudaStream_t, NULL =
 * default stream); the return value reports argument and launch errors only.
 *
 * The first call on each device looks up the scratch array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture. The address is kept for the life of the
 * process: after cudaDeviceReset on a device, do not call this there again.
 * Every call reuses the same array: calls whose
 * kernels may overlap on the GPU (several streams or host threads) race on
 * it and must be serialised by the caller. */
#define POA_NOALLOC_SCRATCH_BYTES (64u << 20)
typedef struct {
    int32_t n_rows;
    const int32_t* in_ptr;    /* [n_rows + 1] */
    const int32_t* in_row;
    const int32_t* in_weight;
    const uint8_t* in_base;
    const uint8_t* base;      /* [n_rows] */
    const int32_t* ind;
    const int32_t* hq;
    const int32_t* hq_loc;
    const int32_t* tq;
    const int32_t* out_ptr;   /* [n_rows + 1] */
    const int32_t* out_row;
} poa_dev_window;
int poa_align_noalloc(const poa_dev_window* w, const uint8_t* q_dev, int32_t qlen, const poa_params* p,
                      int32_t ab_band, int32_t* moves_dev, int32_t moves_cap, int32_t* result_dev, void* stream);

/* Launch shape of the batch kernel (the autotuner's knobs): key 0 = blocks
 * per SM upper bound (the occupancy calculator still caps it), 1 = maximum
 * number of blocks in total (0 = no cap), 2 = shared memory per warp in
 * bytes, a multiple of 16 (row ring, staged records, query,
 * topsort workspace). Takes effect at the next run. */
int poa_batch_config(poa_ctx* ctx, int32_t key, int64_t value);

/* The measured int32 add+max rate of `device` (no counterpart in the
 * reference): one timed launch of independent v = max(v + inc, floor)
 * chains, 2 operations per step, `iters` steps per chain. It is the
 * denominator of the DP's integer roofline. Allocates a small buffer. */
int poa_int_peak(int device, int iters, double* ops_per_s, double* ms);

/* Page-locked host memory (cudaMallocHost) for callers that want the
 * batch copies to run at full PCIe/NVLink-C2C speed; NULL on failure. */
void* poa_alloc_pinned(size_t bytes);
void poa_free_pinned(void* ptr);

/* Counters since poa_create: [0] kernel launches, [1] alignments, [2] band
 * cells, [3] kernel time in microseconds (when timing is on), [4] H2D bytes,
 * [5] D2H bytes. */
int poa_stats(const poa_ctx* ctx, int64_t* out6);
int poa_set_timing(poa_ctx* ctx, int on);

/* One window set over several GPUs (no counterpart in the reference, which
 * runs one graph per process; configurations with independent windows shard
 * across devices with no exchange between them). poa_batch_partition splits
 * windows by estimated cost (bases x (reads + 1)) with the longest-
 * processing-time rule: part[w] in [0, n_parts), part_cost[g] (may be NULL)
 * the summed cost of part g. poa_batch_consensus_multi runs part g on
 * ctxs[g] (one context per device, each on its own host thread) and writes
 * the same outputs as poa_batch_consensus, in input order. Every device gets
 * the whole seq buffer; read_off may point anywhere in it. */
int poa_batch_partition(const int32_t* read_len, const int32_t* win_off, int32_t n_windows, int32_t n_parts,
                        int32_t* part, int64_t* part_cost);
int poa_batch_consensus_multi(poa_ctx** ctxs, int32_t n_ctx, const uint8_t* seq, int64_t seq_bytes,
                              const int64_t* read_off, const int32_t* read_len, int32_t n_reads,
                              const int32_t* win_off, int32_t n_windows, char* cons, int64_t cons_cap,
                              int64_t* cons_off, int32_t* status);

/* ---- learned band proposer (no counterpart in the reference) -----------
 *
 * minipoa allocates each alignment's DP matrices when it runs it
 * (src/align.cpp:1397). The batch engine instead sizes every window's
 * device slot before one persistent launch. The proposer predicts the sizes
 * from minimizer features (k=15, w=10) of each window's reads: a 3-layer
 * 1D convolution (64 channels) plus MLP, BF16 weights, FP32 accumulation,
 * trained on the band statistics of plain runs (poa_batch_read_stats). The
 * plan never changes a band: results are identical with or without it. */
typedef struct poa_proposer poa_proposer;
/* Number of floats in a weight vector: the network parameters, then output
 * mean[4], output std[4], node margin, record-byte margin, spilled
 * row-store entries per row, minimum spill entries. */
int poa_prop_nweights(void);
/* NULL on failure (no CUDA device or no memory). Starts from a fixed random
 * initialisation. */
poa_proposer* poa_prop_create(int device);
void poa_prop_destroy(poa_proposer* p);
const char* poa_prop_last_error(const poa_proposer* p);
int poa_prop_set_weights(poa_proposer* p, const float* w);
int poa_prop_get_weights(poa_proposer* p, float* w);
/* Train on X [n][32 bins][8 channels] (poa_batch_features) against raw
 * targets Y [n][4] per read: new graph nodes per query base, band cells /
 * (DP rows * (qlen + 1)), record bytes per cell, mean band centre / (qlen + 1).
 * Mini-batch Adam on the GPU; per-epoch mean losses to `losses` (may be NULL).
 * The output standardisation is taken from Y; margins stay as set. */
int poa_prop_train(poa_proposer* p, const float* X, const float* Y, int64_t n, int32_t epochs, int32_t batch,
                   float lr, uint64_t seed, float* losses);
/* Raw predictions Y [n][4] for features X [n][32][8]. */
int poa_prop_predict(poa_proposer* p, const float* X, int64_t n, float* Y);
/* Loss (mean squared error of the standardised outputs) and the gradient of
 * every parameter (poa_prop_nweights() - 12 floats, the parameter layout of
 * poa_prop_get_weights) for one batch of 1..4096 reads, without an update:
 * the backward kernels of one training step. */
int poa_prop_gradient(poa_proposer* p, const float* X, const float* Y, int64_t n, float* grad, float* loss);
/* Features of every read of the uploaded batch: n_reads * 32 * 8 floats. */
int poa_batch_features(poa_ctx* ctx, poa_proposer* p, float* X, int64_t cap);
/* Features, prediction and per-window plan on the device, then
 * poa_batch_plan with it: the next poa_batch_run uses the planned slots. */
int poa_batch_propose(poa_ctx* ctx, poa_proposer* p);
/* Let every following poa_batch_run (and poa_batch_consensus) plan its
 * windows with `p` first, inside the timed run; NULL turns it off. The
 * proposer must outlive its use. */
int poa_batch_use_proposer(poa_ctx* ctx, poa_proposer* p);

#ifdef __cplusplus
}
#endif
#endif
