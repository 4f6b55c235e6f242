// dp_model.cpp - TEST-ONLY sequential model of the CUDA DP kernels.
//
// It runs exactly the per-block steps of plain.cuh (pass 1 over predecessors,
// prefix-max scan, finalisation, backtrack records, row store layout, the
// record-driven backtrack) one block at a time on the CPU, using the same
// dp_core.h / dp_rowops.h functions the kernels use. The tests compare it with
// the oracle on every golden case; that validates the kernel formulation
// (scan form of the I recurrence, block masks, compact records) before any
// GPU run. It is never linked into the product library.
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "driver.h"
#include "dp_rowops.h"

using namespace pb;

namespace {

int64_t align16(int64_t x) { return (x + 15) / 16 * 16; }

struct ModelEngine : DpEngine {
    std::vector<int32_t> rs;
    std::vector<uint8_t> tb;

    void align_many(const std::vector<const HostWindow*>& wins, const std::vector<const uint8_t*>& qs,
                    const std::vector<int32_t>& qlens, const std::vector<int32_t>& abs, const Params& p,
                    std::vector<AlignOut>& outs) override {
        outs.assign(wins.size(), AlignOut());
        for (size_t t = 0; t < wins.size(); t++) run(*wins[t], qs[t], qlens[t], abs[t], p, outs[t]);
    }

    void run(const HostWindow& hw, const uint8_t* q, int qlen, int ab, const Params& p, AlignOut& o) {
        const int n = hw.n, m = qlen + 1;
        std::vector<uint8_t> qsb(qs_bytes(qlen));
        make_qs(q, qlen, qsb.data());
        std::vector<RowMeta> meta(n);
        std::vector<int32_t> state((size_t)AB_NSTATE * n);
        std::vector<int32_t> moves(n + m + 8);
        int32_t out[4] = {0, 0, 0, 0};
        DpArgs a;
        a.v = WinView{n, hw.in_ptr.data(), hw.in_row.data(), hw.in_w.data(), hw.in_base.data(), hw.base.data(),
                      hw.ind.data(), hw.hq.data(), hw.hq_loc.data(), hw.tq.data(), hw.out_ptr.data(),
                      hw.out_row.data()};
        a.qs = qsb.data();
        a.qlen = qlen;
        a.ab_band = ab;
        a.f = p.f;
        a.w = p.b + (p.f ? m / p.f : 0);
        a.sc = scoring_of(p);
        a.meta = meta.data();
        a.state = state.data();
        a.moves = moves.data();
        a.moves_cap = (int32_t)moves.size();
        a.out = out;
        // a small ring (4 rows) exercises the ring/spill placement of the kernels;
        // generous capacity: the ring plus every row at full width
        int64_t full_blocks = (int64_t)(m / BLK + 2);
        a.ring_rows = 4;
        a.ring_blocks = (int32_t)std::min<int64_t>(full_blocks, 24);
        rs.assign((size_t)((int64_t)a.ring_rows * a.ring_blocks * 16 + n * full_blocks * 16 + 16), 0);
        tb.assign((size_t)(n * (full_blocks * BLK * 4 + 16) + 16), 0);
        a.rs = rs.data();
        a.rs_cap = (int64_t)rs.size();
        a.tb = tb.data();
        a.tb_cap = (int64_t)tb.size();
        fill(a, m);
        o.status = out[0];
        o.score = out[1];
        o.cells = out[3];
        if (o.status == ST_OK) {
            int32_t nm = 0;
            o.status = backtrack_records(a, m, nm);
            o.moves.assign(moves.begin(), moves.begin() + nm);
        }
    }

    static void fill(DpArgs& a, int m) {
        const int n = a.v.n;
        const Scoring sc = a.sc;
        const bool adaptive = a.f > 0 && a.ab_band;
        if (adaptive)
            for (int r = 0; r < n; r++) adaptive_init_entry(a, r, m);
        int64_t st_next = a.ring_rows > 0 ? (int64_t)a.ring_rows * a.ring_blocks * 16 : 0;
        int64_t tb_next = 0, cells = 0;
        std::vector<int32_t> H0, Dk, Mf, If;
        for (int i = 0; i < n; i++) {
            int Bs, Be;
            row_band(a, i, m, Bs, Be);
            if (i == 0) Bs = 0;  // row 0 always starts at column 0 (Ms[0] = 0)
            const int bn = Be - Bs - 1;
            if (bn < 0) { a.out[0] = ST_DEGENERATE; return; }
            const int e0 = a.v.in_ptr[i], d = i == 0 ? 0 : a.v.in_ptr[i + 1] - e0;
            if (d > MAX_MULTI_PRED) { a.out[0] = ST_INDEGREE; return; }
            const int bpc = d >= 2 ? 4 : 1;
            int64_t row_st = st_next;
            bool linear = true;
            if (a.ring_rows > 0) {
                int maxs = i;
                for (int e = a.v.out_ptr[i]; e < a.v.out_ptr[i + 1]; e++) maxs = std::max(maxs, a.v.out_row[e]);
                if (!((maxs - i >= a.ring_rows) || (bn > a.ring_blocks))) {
                    row_st = (int64_t)(i % a.ring_rows) * a.ring_blocks * 16;
                    linear = false;
                }
            }
            RowMeta rm{Bs, Be, row_st, tb_next};
            if ((linear && row_st + (int64_t)bn * 16 > a.rs_cap) || tb_next + (int64_t)bn * BLK * bpc > a.tb_cap) {
                a.out[0] = ST_OOM;
                return;
            }
            if (linear) st_next = row_st + (int64_t)bn * 16;
            a.meta[i] = rm;
            cells += (int64_t)bn * BLK;
            H0.assign((size_t)bn * BLK, 0);
            Dk.assign((size_t)bn * BLK, 0);
            Mf.assign((size_t)bn * BLK, 0);
            If.assign((size_t)bn * BLK, 0);
            // pass 1
            for (int b = 0; b < bn; b++) {
                const int B = Bs + b;
                int32_t Mpre[BLK], Dv[BLK];
                for (int l = 0; l < BLK; l++) Mpre[l] = Dv[l] = NEG_INF;
                if (i == 0) {
                    for (int l = 0; l < BLK; l++) Mpre[l] = (b * BLK + l == 0) ? 0 : NEG_INF;
                }
                const uint8_t* qc8 = a.qs + (int64_t)B * BLK;
                for (int e = e0; e < e0 + d; e++) {
                    const int pr = a.v.in_row[e];
                    const RowMeta pm = a.meta[pr];
                    PredMask mk = pred_mask(B, pm.Bs, pm.Be);
                    const int32_t* Mb = a.rs + pm.st + (int64_t)(B - pm.Bs) * 16;
                    int32_t mprev = mk.prev_in ? a.rs[pm.st + (int64_t)(B - 1 - pm.Bs) * 16 + 7] : NEG_INF;
                    if (mk.blk_in) pass1_pred(sc, mk, b == 0, a.v.in_base[e], Mb, Mb + 8, mprev, qc8, Mpre, Dv);
                }
                for (int l = 0; l < BLK; l++) {
                    H0[b * BLK + l] = mx(Mpre[l], Dv[l]);
                    Dk[b * BLK + l] = Dv[l];
                }
            }
            // scan + finalise (row 0: M = H0 exactly, I = NEG_INF)
            int32_t P = 0;
            for (int b = 0; b < bn; b++) {
                int32_t* M = &Mf[b * BLK];
                int32_t* I = &If[b * BLK];
                if (i == 0) {
                    for (int l = 0; l < BLK; l++) { M[l] = H0[b * BLK + l]; I[l] = NEG_INF; }
                } else {
                    finalize_block(sc, b * BLK, P, &H0[b * BLK], M, I);
                    // the single-alignment kernels derive a warp's left neighbour
                    // from the scan summary alone; it must equal the full block
                    int32_t k06 = scan_key(H0[b * BLK], b * BLK, sc.e1), M7, I7;
                    for (int l = 1; l < BLK - 1; l++) k06 = mx(k06, scan_key(H0[b * BLK + l], b * BLK + l, sc.e1));
                    finalize_last(sc, b * BLK, P, k06, H0[b * BLK + BLK - 1], M7, I7);
                    if (M7 != M[BLK - 1] || I7 != I[BLK - 1]) { a.out[0] = ST_BAD_ARG; return; }
                }
                for (int l = 0; l < BLK; l++) {
                    int32_t key = scan_key(H0[b * BLK + l], b * BLK + l, sc.e1);
                    P = (b == 0 && l == 0) ? key : mx(P, key);
                }
            }
            // records + store
            for (int b = 0; b < bn; b++) {
                const int B = Bs + b;
                const int32_t* M = &Mf[b * BLK];
                const int32_t* I = &If[b * BLK];
                const int32_t* D = &Dk[b * BLK];
                const uint8_t* qc8 = a.qs + (int64_t)B * BLK;
                FlagAcc acc;
                flag_acc_init(acc);
                for (int e = e0; e < e0 + d; e++) {
                    const int pr = a.v.in_row[e];
                    const RowMeta pm = a.meta[pr];
                    PredMask mk = pred_mask(B, pm.Bs, pm.Be);
                    const int32_t* Mb = a.rs + pm.st + (int64_t)(B - pm.Bs) * 16;
                    int32_t mprev = mk.prev_in ? a.rs[pm.st + (int64_t)(B - 1 - pm.Bs) * 16 + 7] : NEG_INF;
                    if (mk.blk_in || mk.prev_in)
                        flags_pred(sc, mk, a.v.in_base[e], a.v.in_w[e], e - e0, Mb, Mb + 8, mprev, qc8, M, D, acc);
                }
                int32_t* dst = a.rs + rm.st + (int64_t)b * 16;
                for (int l = 0; l < BLK; l++) {
                    const int j = b * BLK + l;
                    int32_t Ml = j > 0 ? Mf[j - 1] : NEG_INF, Il = j > 0 ? If[j - 1] : NEG_INF;
                    uint32_t own = own_flags(sc, j, M[l], D[l], I[l], Ml, Il);
                    if (bpc == 1) a.tb[rm.tb + j] = encode_small(own, acc, l, a.v.ind[i]);
                    else *(uint32_t*)(a.tb + rm.tb + (int64_t)j * 4) = encode_wide(own, acc, l, a.v.ind[i]);
                    dst[l] = M[l];
                    dst[8 + l] = D[l];
                }
            }
            if (adaptive && i >= 1) {
                int max_j = 0;
                for (int j = 1; j < bn * BLK; j++) max_j = Mf[j] > Mf[max_j] ? j : max_j;
                adaptive_update(a, i, Bs, max_j);
            }
            tb_next = align16(tb_next + (int64_t)bn * BLK * bpc);
        }
        const RowMeta last = a.meta[n - 1];
        const int jm = m - last.Bs * BLK;
        a.out[1] = a.rs[last.st + (int64_t)(jm / BLK) * 16 + jm % BLK];
        a.out[3] = (int32_t)std::min<int64_t>(cells, INT32_MAX);
        a.out[0] = ST_OK;
    }
};

}  // namespace

extern "C" {

// Run the whole driver with the model engine. params: match, mismatch,
// gap_open, gap_ext, b, f, ab_band, result, seeding. Returns status; *text is malloc'd.
int model_run_gfa(int nseq, const char* const* seqs, const int* lens, const int* params, const char* gfa,
                  int gfa_len, const char* const* hdrs, char** text, int* scores, int scores_cap);

int model_run(int nseq, const char* const* seqs, const int* lens, const int* params, char** text,
              int* scores, int scores_cap) {
    return model_run_gfa(nseq, seqs, lens, params, nullptr, -1, nullptr, text, scores, scores_cap);
}

// gfa_len < 0: no graph file (plain run); hdrs may be null
int model_run_gfa(int nseq, const char* const* seqs, const int* lens, const int* params, const char* gfa,
                  int gfa_len, const char* const* hdrs, char** text, int* scores, int scores_cap) {
    Params p;
    p.match = params[0]; p.mismatch = params[1]; p.gap_open1 = params[2]; p.gap_ext1 = params[3];
    p.b = params[4]; p.f = params[5]; p.ab_band = params[6]; p.result = params[7]; p.enable_seeding = params[8];
    p.progressive = params[9];
    normalize_params(p);
    std::vector<std::string> s(nseq), headers;
    for (int i = 0; i < nseq; i++) s[i].assign(seqs[i], lens[i]);
    if (hdrs)
        for (int i = 0; i < nseq; i++) headers.push_back(hdrs[i] ? hdrs[i] : "");
    ModelEngine eng;
    std::string out;
    std::vector<int32_t> sc;
    std::string g;
    if (gfa_len >= 0) g.assign(gfa ? gfa : "", (size_t)gfa_len);
    int st = run_reads(p, s, headers, eng, out, &sc, nullptr, gfa_len >= 0 ? &g : nullptr);
    *text = (char*)malloc(out.size() + 1);
    memcpy(*text, out.data(), out.size());
    (*text)[out.size()] = 0;
    if (scores)
        for (size_t i = 0; i < sc.size() && (int)i < scores_cap; i++) scores[i] = sc[i];
    return st;
}

void model_free(void* p) { free(p); }

// finalize_last against finalize_block on random blocks: H0 values from the
// whole int32 range near NEG_INF up to large scores, random prefixes P and
// block positions, several scorings. Returns the number of mismatches.
int model_check_finalize_last(uint64_t seed, int iters) {
    uint64_t x = seed * 0x9E3779B97F4A7C15ull + 1;
    auto rnd = [&x]() {
        x ^= x << 13; x ^= x >> 7; x ^= x << 17;
        return x;
    };
    const int32_t pool[] = {NEG_INF, NEG_INF + 1, NEG_INF + 7, -1000000, -5, 0, 3, 1000000, 0x3f3f3f3f};
    int bad = 0;
    for (int it = 0; it < iters; it++) {
        Scoring sc;
        sc.match = (int32_t)(rnd() % 5);
        sc.mismatch = -(int32_t)(rnd() % 7);
        const int32_t e1 = -(int32_t)(1 + rnd() % 4);
        sc.e1 = e1;
        sc.o1 = e1 - (int32_t)(rnd() % 8);  // o1 <= e1, as the prefix-max form requires
        const int j0 = (int)(rnd() % 3 == 0 ? 0 : (rnd() % 4096) * BLK);
        int32_t H0[BLK];
        for (int l = 0; l < BLK; l++)
            H0[l] = rnd() % 3 == 0 ? pool[rnd() % 9] : (int32_t)(rnd() % 4000000) - 2000000;
        const int32_t P = rnd() % 4 == 0 ? pool[rnd() % 9] : (int32_t)(rnd() % 4000000) - 2000000;
        int32_t M[BLK], I[BLK], M7, I7;
        finalize_block(sc, j0, P, H0, M, I);
        int32_t k06 = scan_key(H0[0], j0, sc.e1);
        for (int l = 1; l < BLK - 1; l++) k06 = mx(k06, scan_key(H0[l], j0 + l, sc.e1));
        finalize_last(sc, j0, P, k06, H0[BLK - 1], M7, I7);
        if (M7 != M[BLK - 1] || I7 != I[BLK - 1]) bad++;
    }
    return bad;
}
}
