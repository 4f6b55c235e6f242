// capi.cpp - the extern "C" boundary (include/poa_b200.h). No exception or
// C++ type crosses it: failures become status codes plus a per-context
// message.
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

#include "../../include/poa_b200.h"
#include <cuda_runtime.h>

#include "batch.h"
#include "gpu_engine.h"
#include "proposer.h"

struct poa_ctx {
    int device = 0;
    pb::Params p;
    pb::GpuEngine* eng = nullptr;
    pb::BatchEngine* batch = nullptr;
    std::string err;
};

struct poa_proposer {
    int device = 0;
    pb::Proposer* prop = nullptr;
    std::string err;
};

namespace {

constexpr int kPropK = pb::PROP_K, kPropW = pb::PROP_W;

int prop_fail(poa_proposer* p, int code, const std::string& msg) {
    if (p) p->err = msg;
    return code;
}

pb::Params to_params(const poa_params* c) {
    pb::Params p;
    p.match = c->match;
    p.mismatch = c->mismatch;
    p.gap_open1 = c->gap_open;
    p.gap_ext1 = c->gap_ext;
    p.b = c->band_b;
    p.f = c->band_f;
    p.ab_band = c->ab_band;
    p.enable_seeding = c->seeding;
    p.k = c->k;
    p.mm_w = c->mm_w;
    p.poa_w = c->poa_w;
    p.thread = c->thread;
    p.result = c->result;
    p.progressive = c->progressive;
    p.verbose = c->verbose;
    pb::normalize_params(p);
    return p;
}

int fail(poa_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

// Window view of ranks [rank(beg), rank(end)] straight from the flat graph.
void window_from_view(const poa_graph_view& g, int beg_id, int end_id, bool with_lens, pb::HostWindow& w) {
    const int beg_i = g.rank[beg_id], end_i = g.rank[end_id];
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
        const int u = g.rank_to_id[beg_i + r];
        w.row_node[r] = u;
        w.base[r] = g.base[u];
        w.ind[r] = g.ind[u];
        if (with_lens) {
            w.hq[r] = g.hlen[beg_i + r] - g.hlen[beg_i];
            w.hq_loc[r] = g.hlen[r] - g.hlen[beg_i];
            w.tq[r] = g.tlen[beg_i + r] - g.tlen[end_i];
        }
        int deg = 0;
        for (int e = g.in_ptr[u]; e < g.in_ptr[u + 1]; e++) {
            int p = g.rank[g.in_id[e]] - beg_i;
            if (p < 0) continue;
            w.in_row.push_back(p);
            w.in_w.push_back(g.in_weight[e]);
            w.in_base.push_back(p == 0 ? 4 : g.base[g.in_id[e]]);
            deg++;
        }
        if (deg > w.max_indeg) w.max_indeg = deg;
        w.in_ptr[r + 1] = (int32_t)w.in_row.size();
        for (int e = g.out_ptr[u]; e < g.out_ptr[u + 1]; e++) {
            int s = g.rank[g.out_id[e]] - beg_i;
            if (s >= n) continue;
            w.out_row.push_back(s);
        }
        w.out_ptr[r + 1] = (int32_t)w.out_row.size();
    }
}

}  // namespace

extern "C" {

void poa_params_init(poa_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->match = 2; p->mismatch = -4; p->gap_open = -4; p->gap_ext = -2;
    p->band_b = 100; p->band_f = 40;
    p->k = 19; p->mm_w = 10; p->poa_w = 0;
    p->thread = 1;
}

const char* poa_status_str(int s) {
    switch (s) {
        case POA_OK: return "ok";
        case POA_BAND_ESCAPE: return "backtrack left the band";
        case POA_BT_FAIL: return "backtrack error";
        case POA_BAD_ARG: return "bad argument";
        case POA_OOM: return "out of device memory";
        case POA_INDEGREE: return "node in-degree above 510 within one window";
        case POA_DEGENERATE: return "degenerate band or sub-window";
        case POA_CAPACITY: return "window outgrew its device capacity";
        case POA_CUDA: return "CUDA error";
        case POA_UNSUPPORTED: return "unsupported option";
        default: return "unknown status";
    }
}

poa_ctx* poa_create(int device, const poa_params* p) {
    poa_ctx* ctx = new (std::nothrow) poa_ctx;
    if (!ctx) return nullptr;
    try {
        poa_params d;
        poa_params_init(&d);
        ctx->p = to_params(p ? p : &d);
        ctx->device = device;
        ctx->eng = new pb::GpuEngine(device);
    } catch (const std::exception& e) {
        delete ctx->eng;
        delete ctx;
        return nullptr;
    }
    return ctx;
}

void poa_destroy(poa_ctx* ctx) {
    if (!ctx) return;
    delete ctx->batch;
    delete ctx->eng;
    delete ctx;
}

const char* poa_last_error(const poa_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void poa_free(void* ptr) { std::free(ptr); }

int poa_align(poa_ctx* ctx, const poa_graph_view* g, int32_t beg_id, int32_t end_id, const uint8_t* q_enc,
              int32_t qlen, int32_t ab_band, poa_res* out, int32_t out_cap, int32_t* out_len, int32_t* score) {
    if (!ctx || !g || (!q_enc && qlen > 0) || qlen < 0 || !out || !out_len || !score)
        return fail(ctx, POA_BAD_ARG, "null argument");
    if (beg_id < 0 || end_id < 0 || beg_id >= g->n_nodes || end_id >= g->n_nodes)
        return fail(ctx, POA_BAD_ARG, "node id out of range");
    try {
        pb::HostWindow w;
        const bool lens = ctx->p.f > 0;
        if (lens && (!g->hlen || !g->tlen)) return fail(ctx, POA_BAD_ARG, "hlen/tlen required when band_f > 0");
        window_from_view(*g, beg_id, end_id, lens, w);
        if (w.n <= 0) return fail(ctx, POA_DEGENERATE, "end rank precedes begin rank");
        std::vector<pb::AlignOut> outs;
        ctx->eng->align_many({&w}, {q_enc}, {qlen}, {ab_band}, ctx->p, outs);
        if (outs[0].status != POA_OK) return fail(ctx, outs[0].status, poa_status_str(outs[0].status));
        const std::vector<int32_t>& mv = outs[0].moves;
        if ((int32_t)mv.size() > out_cap) return fail(ctx, POA_BAD_ARG, "output capacity too small");
        int k = 0;
        for (int t = (int)mv.size() - 1; t >= 0; t--, k++) {
            const int kind = pb::mv_kind(mv[t]), qc = pb::mv_qc(mv[t]);
            poa_res r;
            r.base = (uint8_t)qc;
            r.from = -1;
            r.aligned_id = -1;
            if (kind != pb::MV_INSERT) {
                const int pre = w.row_node[pb::mv_row(mv[t])];
                if (kind == pb::MV_MATCH) {
                    r.from = pre;
                    r.base = g->base[pre];
                } else {
                    const int par = g->par_id[pre];
                    const int al = g->aligned[par * 5 + qc];
                    if (al != -1) r.from = al;
                    else r.aligned_id = par;
                }
            }
            out[k] = r;
        }
        *out_len = k;
        *score = outs[0].score;
        return POA_OK;
    } catch (const std::exception& e) {
        return fail(ctx, POA_CUDA, e.what());
    }
}

namespace {

int run_impl(poa_ctx* ctx, const std::string* gfa, int32_t nseq, const char* const* seqs, const int32_t* lens,
             const char* const* headers, char** text, size_t* text_len, int32_t* scores) {
    if (!ctx || nseq < 0 || (nseq > 0 && (!seqs || !lens)) || !text) return fail(ctx, POA_BAD_ARG, "null argument");
    try {
        std::vector<std::string> s(nseq), h;
        for (int i = 0; i < nseq; i++) {
            if (lens[i] < 0 || (lens[i] > 0 && !seqs[i])) return fail(ctx, POA_BAD_ARG, "bad sequence");
            s[i].assign(seqs[i] ? seqs[i] : "", (size_t)lens[i]);
        }
        if (headers) {
            h.resize(nseq);
            for (int i = 0; i < nseq; i++) h[i] = headers[i] ? headers[i] : "";
        }
        std::string out;
        std::vector<int32_t> sc;
        int st = pb::run_reads(ctx->p, s, h, *ctx->eng, out, scores ? &sc : nullptr, nullptr, gfa);
        if (st != POA_OK) return fail(ctx, st, out.empty() ? std::string(poa_status_str(st)) : out);
        char* buf = (char*)std::malloc(out.size() + 1);
        if (!buf) return fail(ctx, POA_BAD_ARG, "host allocation failed");
        std::memcpy(buf, out.data(), out.size());
        buf[out.size()] = 0;
        *text = buf;
        if (text_len) *text_len = out.size();
        if (scores) {
            // one entry per read: reads whose alignment ran on an empty graph get 0
            int first_dp = nseq - (int)sc.size();
            for (int i = 0; i < nseq; i++) scores[i] = i >= first_dp ? sc[i - first_dp] : 0;
        }
        return POA_OK;
    } catch (const std::exception& e) {
        return fail(ctx, POA_CUDA, e.what());
    }
}

}  // namespace

int poa_run(poa_ctx* ctx, int32_t nseq, const char* const* seqs, const int32_t* lens,
            const char* const* headers, char** text, size_t* text_len, int32_t* scores) {
    return run_impl(ctx, nullptr, nseq, seqs, lens, headers, text, text_len, scores);
}

int poa_run_gfa(poa_ctx* ctx, const char* gfa, size_t gfa_len, int32_t nseq, const char* const* seqs,
                const int32_t* lens, const char* const* headers, char** text, size_t* text_len, int32_t* scores) {
    if (!gfa && gfa_len > 0) return fail(ctx, POA_BAD_ARG, "null GFA text");
    std::string g;
    try {
        g.assign(gfa ? gfa : "", gfa_len);
    } catch (const std::exception& e) {
        return fail(ctx, POA_OOM, e.what());
    }
    return run_impl(ctx, &g, nseq, seqs, lens, headers, text, text_len, scores);
}

int poa_batch_upload(poa_ctx* ctx, const uint8_t* seq, int64_t seq_bytes, const int64_t* read_off,
                     const int32_t* read_len, int32_t n_reads, const int32_t* win_off, int32_t n_windows) {
    if (!ctx || (seq_bytes > 0 && !seq) || n_reads < 0 || n_windows < 0 || (n_reads > 0 && (!read_off || !read_len)) ||
        !win_off)
        return fail(ctx, POA_BAD_ARG, "null argument");
    if (win_off[0] != 0 || win_off[n_windows] != n_reads) return fail(ctx, POA_BAD_ARG, "win_off must span all reads");
    for (int32_t w = 0; w < n_windows; w++)
        if (win_off[w + 1] < win_off[w]) return fail(ctx, POA_BAD_ARG, "win_off must be non-decreasing");
    for (int32_t r = 0; r < n_reads; r++)
        if (read_len[r] < 0 || read_off[r] < 0 || read_off[r] + read_len[r] > seq_bytes)
            return fail(ctx, POA_BAD_ARG, "read outside seq");
    if (ctx->p.enable_seeding || ctx->p.progressive || ctx->p.result != 0)
        return fail(ctx, POA_UNSUPPORTED, "batched windows run the consensus mode without -S/-p");
    try {
        if (!ctx->batch) ctx->batch = new pb::BatchEngine(ctx->device);
        pb::BatchInput in{seq, seq_bytes, read_off, read_len, n_reads, win_off, n_windows};
        ctx->batch->upload(in, ctx->p);
        return POA_OK;
    } catch (const std::exception& e) {
        return fail(ctx, POA_CUDA, e.what());
    }
}

int poa_batch_run(poa_ctx* ctx, double* device_ms) {
    if (!ctx || !ctx->batch) return fail(ctx, POA_BAD_ARG, "nothing uploaded");
    try {
        ctx->batch->run();
        if (device_ms) *device_ms = ctx->batch->stats.run_ms;
        return POA_OK;
    } catch (const std::exception& e) {
        return fail(ctx, POA_CUDA, e.what());
    }
}

int poa_batch_download(poa_ctx* ctx, char* cons, int64_t cons_cap, int64_t* cons_off, int32_t* status) {
    if (!ctx || !ctx->batch || !cons_off || !status) return fail(ctx, POA_BAD_ARG, "null argument");
    try {
        std::vector<std::string> c;
        std::vector<int32_t> st;
        ctx->batch->download(c, st);
        int64_t pos = 0;
        for (size_t w = 0; w < c.size(); w++) {
            cons_off[w] = pos;
            if (pos + (int64_t)c[w].size() > cons_cap) return fail(ctx, POA_BAD_ARG, "consensus buffer too small");
            if (!c[w].empty()) std::memcpy(cons + pos, c[w].data(), c[w].size());
            pos += (int64_t)c[w].size();
            status[w] = st[w];
        }
        cons_off[c.size()] = pos;
        return POA_OK;
    } catch (const std::exception& e) {
        return fail(ctx, POA_CUDA, e.what());
    }
}

int poa_batch_consensus(poa_ctx* ctx, const uint8_t* seq, int64_t seq_bytes, const int64_t* read_off,
                        const int32_t* read_len, int32_t n_reads, const int32_t* win_off, int32_t n_windows,
                        char* cons, int64_t cons_cap, int64_t* cons_off, int32_t* status) {
    int st = poa_batch_upload(ctx, seq, seq_bytes, read_off, read_len, n_reads, win_off, n_windows);
    if (st != POA_OK) return st;
    st = poa_batch_run(ctx, nullptr);
    if (st != POA_OK) return st;
    return poa_batch_download(ctx, cons, cons_cap, cons_off, status);
}

int poa_batch_stats(poa_ctx* ctx, int64_t* o) {
    if (!ctx || !ctx->batch || !o) return POA_BAD_ARG;
    try {
        ctx->batch->sync_stats();
    } catch (const std::exception& e) {
        return fail(ctx, POA_CUDA, e.what());
    }
    const pb::BatchStats& s = ctx->batch->stats;
    o[0] = s.cells; o[1] = s.failed; o[2] = s.slots; o[3] = s.slot_bytes; o[4] = s.h2d_bytes; o[5] = s.d2h_bytes;
    for (int k = 0; k < 6; k++) o[6 + k] = s.phase_cycles[k];
    o[12] = s.launches;
    o[13] = s.retried;
    o[14] = s.fallback;
    o[15] = (int64_t)(s.kernel_ms * 1000.0);
    o[16] = (int64_t)(s.run_ms * 1000.0);
    o[17] = (int64_t)(s.plan_ms * 1000.0);
    o[18] = s.edge_cells;
    return POA_OK;
}

int poa_batch_plan(poa_ctx* ctx, const int32_t* nodes, const int64_t* tb_bytes, const int64_t* spill,
                   const float* cost) {
    if (!ctx || !ctx->batch) return fail(ctx, POA_BAD_ARG, "no uploaded batch");
    if (nodes && (!tb_bytes || !spill || !cost)) return fail(ctx, POA_BAD_ARG, "incomplete plan");
    try {
        ctx->batch->set_plan(nodes, tb_bytes, spill, cost);
    } catch (const std::exception& e) {
        return fail(ctx, POA_OOM, e.what());
    }
    return POA_OK;
}

int poa_batch_plan_get(poa_ctx* ctx, int32_t* nodes, int64_t* tb_bytes, int64_t* spill, int32_t n_windows) {
    if (!ctx || !ctx->batch || !nodes || !tb_bytes || !spill) return fail(ctx, POA_BAD_ARG, "null argument");
    const pb::BatchEngine& b = *ctx->batch;
    if (b.plan_nodes().empty()) return fail(ctx, POA_BAD_ARG, "the last run had no plan");
    if ((size_t)n_windows != b.plan_nodes().size()) return fail(ctx, POA_BAD_ARG, "window count differs from the plan");
    for (int32_t w = 0; w < n_windows; w++) {
        nodes[w] = b.plan_nodes()[w];
        tb_bytes[w] = b.plan_tb()[w];
        spill[w] = b.plan_spill()[w];
    }
    return POA_OK;
}

int poa_batch_config(poa_ctx* ctx, int32_t key, int64_t value) {
    if (!ctx) return POA_BAD_ARG;
    try {
        if (!ctx->batch) ctx->batch = new pb::BatchEngine(ctx->device);
    } catch (const std::exception& e) {
        return fail(ctx, POA_CUDA, e.what());
    }
    switch (key) {
        case 0: if (value < 1 || value > 32) return fail(ctx, POA_BAD_ARG, "blocks per SM"); ctx->batch->blocks_per_sm = (int32_t)value; break;
        case 1: if (value < 0) return fail(ctx, POA_BAD_ARG, "max blocks"); ctx->batch->max_blocks = (int32_t)value; break;
        case 2:
            if (value < 1024 || value > 48 * 1024 || value % 16 != 0)
                return fail(ctx, POA_BAD_ARG, "smem per warp: 1024..49152 bytes, a multiple of 16");
            ctx->batch->smem_per_warp = (int32_t)value;
            break;
        default: return fail(ctx, POA_BAD_ARG, "unknown key");
    }
    return POA_OK;
}

void* poa_alloc_pinned(size_t bytes) {
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes ? bytes : 1) != cudaSuccess) return nullptr;
    return p;
}

void poa_free_pinned(void* ptr) {
    if (ptr) cudaFreeHost(ptr);
}

int poa_batch_read_stats(poa_ctx* ctx, int32_t* out, int64_t cap) {
    if (!ctx || !ctx->batch || !out) return fail(ctx, POA_BAD_ARG, "null argument");
    try {
        std::vector<int32_t> v;
        ctx->batch->read_stats(v);
        if ((int64_t)v.size() > cap) return fail(ctx, POA_BAD_ARG, "read stats buffer too small");
        std::memcpy(out, v.data(), 4 * v.size());
        return POA_OK;
    } catch (const std::exception& e) {
        return fail(ctx, POA_CUDA, e.what());
    }
}

int poa_stats(const poa_ctx* ctx, int64_t* o) {
    if (!ctx || !o) return POA_BAD_ARG;
    const pb::EngineStats& s = ctx->eng->stats;
    o[0] = s.launches; o[1] = s.alignments; o[2] = s.cells;
    o[3] = (int64_t)(s.kernel_ms * 1000.0); o[4] = s.h2d_bytes; o[5] = s.d2h_bytes;
    return POA_OK;
}

int poa_set_timing(poa_ctx* ctx, int on) {
    if (!ctx) return POA_BAD_ARG;
    ctx->eng->timing = on != 0;
    return POA_OK;
}


/* ---- learned band proposer ---------------------------------------------- */

int poa_prop_nweights(void) { return pb::PROP_NWEIGHTS; }

poa_proposer* poa_prop_create(int device) {
    poa_proposer* p = new poa_proposer();
    p->device = device;
    try {
        p->prop = new pb::Proposer(device);
    } catch (const std::exception&) {
        delete p;
        return nullptr;
    }
    return p;
}

void poa_prop_destroy(poa_proposer* p) {
    if (!p) return;
    delete p->prop;
    delete p;
}

const char* poa_prop_last_error(const poa_proposer* p) { return p ? p->err.c_str() : "null proposer"; }

int poa_prop_set_weights(poa_proposer* p, const float* w) {
    if (!p || !w) return prop_fail(p, POA_BAD_ARG, "null argument");
    try {
        p->prop->set_weights(w);
    } catch (const std::invalid_argument& e) {
        return prop_fail(p, POA_BAD_ARG, e.what());
    } catch (const std::exception& e) {
        return prop_fail(p, POA_CUDA, e.what());
    }
    return POA_OK;
}

int poa_prop_get_weights(poa_proposer* p, float* w) {
    if (!p || !w) return prop_fail(p, POA_BAD_ARG, "null argument");
    try {
        p->prop->get_weights(w);
    } catch (const std::exception& e) {
        return prop_fail(p, POA_CUDA, e.what());
    }
    return POA_OK;
}

int poa_prop_train(poa_proposer* p, const float* X, const float* Y, int64_t n, int32_t epochs, int32_t batch,
                   float lr, uint64_t seed, float* losses) {
    if (!p || !X || !Y) return prop_fail(p, POA_BAD_ARG, "null argument");
    if (n <= 0 || epochs <= 0 || batch <= 0 || batch > 4096 || !(lr > 0.f))
        return prop_fail(p, POA_BAD_ARG, "bad training arguments");
    try {
        p->prop->train(X, Y, n, epochs, batch, lr, seed, losses);
    } catch (const std::exception& e) {
        return prop_fail(p, POA_CUDA, e.what());
    }
    return POA_OK;
}

int poa_prop_gradient(poa_proposer* p, const float* X, const float* Y, int64_t n, float* grad, float* loss) {
    if (!p || !X || !Y || !grad) return prop_fail(p, POA_BAD_ARG, "null argument");
    if (n <= 0 || n > 4096) return prop_fail(p, POA_BAD_ARG, "gradient batch must hold 1..4096 reads");
    try {
        const float l = p->prop->gradient(X, Y, n, grad);
        if (loss) *loss = l;
    } catch (const std::exception& e) {
        return prop_fail(p, POA_CUDA, e.what());
    }
    return POA_OK;
}

int poa_prop_predict(poa_proposer* p, const float* X, int64_t n, float* Y) {
    if (!p || (n > 0 && (!X || !Y)) || n < 0) return prop_fail(p, POA_BAD_ARG, "bad argument");
    if (n == 0) return POA_OK;
    try {
        p->prop->predict_host(X, n, Y);
    } catch (const std::exception& e) {
        return prop_fail(p, POA_CUDA, e.what());
    }
    return POA_OK;
}

int poa_batch_features(poa_ctx* ctx, poa_proposer* p, float* X, int64_t cap) {
    if (!ctx || !ctx->batch || !p || !X) return fail(ctx, POA_BAD_ARG, "null argument or no uploaded batch");
    try {
        const pb::DeviceWindows dw = ctx->batch->device_windows();
        const int64_t need = (int64_t)dw.n_reads * pb::PROP_BINS * pb::PROP_CIN;
        if (need > cap) return fail(ctx, POA_BAD_ARG, "feature buffer too small");
        if (need == 0) return POA_OK;
        float* d = nullptr;
        pb::cuda_check(cudaMalloc(&d, 4 * (size_t)need), "cudaMalloc(features)");
        p->prop->features(dw, kPropK, kPropW, d, dw.stream);
        const cudaError_t e1 = cudaMemcpyAsync(X, d, 4 * (size_t)need, cudaMemcpyDeviceToHost, (cudaStream_t)dw.stream);
        const cudaError_t e2 = cudaStreamSynchronize((cudaStream_t)dw.stream);
        cudaFree(d);
        pb::cuda_check(e1 != cudaSuccess ? e1 : e2, "D2H features");
    } catch (const std::exception& e) {
        return fail(ctx, POA_CUDA, e.what());
    }
    return POA_OK;
}

int poa_batch_use_proposer(poa_ctx* ctx, poa_proposer* p) {
    if (!ctx) return POA_BAD_ARG;
    try {
        if (!ctx->batch) ctx->batch = new pb::BatchEngine(ctx->device);
    } catch (const std::exception& e) {
        return fail(ctx, POA_CUDA, e.what());
    }
    ctx->batch->set_proposer(p ? p->prop : nullptr);
    return POA_OK;
}

int poa_batch_propose(poa_ctx* ctx, poa_proposer* p) {
    if (!ctx || !ctx->batch || !p) return fail(ctx, POA_BAD_ARG, "null argument or no uploaded batch");
    try {
        std::vector<int32_t> nodes;
        std::vector<int64_t> tb, spill;
        std::vector<float> cost;
        p->prop->plan(ctx->batch->device_windows(), kPropK, kPropW, nodes, tb, spill, cost);
        ctx->batch->set_plan(nodes.data(), tb.data(), spill.data(), cost.data());
    } catch (const std::exception& e) {
        return fail(ctx, POA_CUDA, e.what());
    }
    return POA_OK;
}

}  // extern "C"
