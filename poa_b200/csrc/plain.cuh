// plain.cuh - the single-alignment DP kernel for sm_100a: one CTA per poa()
// call (src/align.cpp:1353-1737), integer-only, no tensor cores.
//
// Work mapping. Row i (rank beg+i) covers absolute column blocks [Bs, Be-1);
// thread t of the CTA owns block Bs + c*NT + t of chunk c (rows wider than
// the CTA are processed in chunks, the scan carrying across chunks).
//   1. pass 1: for every in-window predecessor p (in-list order) the thread
//      loads p's M/D block (64 B, coalesced across the CTA) plus one M cell to
//      its left, and folds the diagonal and vertical terms (pass1_pred).
//   2. the horizontal gap recurrence is a CTA-wide exclusive prefix max of
//      H0[k] - k*e1 (warp shuffles + one barrier, CtaGroup::scan).
//   3. final M and I, the backtrack records of the block (own-row tests plus
//      one comparison sweep over the predecessors; the left neighbour of a
//      warp's first block comes from the scan summary), and the row's M/D
//      blocks are written back to global memory, all 16-byte vector stores.
//   4. with the adaptive band, a CTA argmax of M, then warp 0 propagates
//      the band state to the successors (src/align.cpp:1516-1568), one lane
//      per edge, from inputs it copied with cp.async when the row started;
//      thread 0 then prepares the next row's header.
// After the last row thread 0 walks the records back from (n-1, m).
// This kernel serves adaptive-band calls (-B, -S sub-windows); static-band
// calls run k_plain_static (plain_static.cuh).
#pragma once
#include <climits>

#include "dp_rowops.h"

namespace pb {

__device__ __forceinline__ int32_t warp_incl_max(int32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int32_t y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v = mx(v, y);
    }
    return v;
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long y = __shfl_xor_sync(0xffffffffu, v, o);
        v = y > v ? y : v;
    }
    return v;
}

__device__ __forceinline__ void load_block16(const int32_t* src, int32_t* Mb, int32_t* Db) {
    const int4* p = reinterpret_cast<const int4*>(src);
    int4 a = p[0], b = p[1], c = p[2], d = p[3];
    Mb[0] = a.x; Mb[1] = a.y; Mb[2] = a.z; Mb[3] = a.w;
    Mb[4] = b.x; Mb[5] = b.y; Mb[6] = b.z; Mb[7] = b.w;
    Db[0] = c.x; Db[1] = c.y; Db[2] = c.z; Db[3] = c.w;
    Db[4] = d.x; Db[5] = d.y; Db[6] = d.z; Db[7] = d.w;
}

__device__ __forceinline__ void store_block16(int32_t* dst, const int32_t* M, const int32_t* D) {
    int4* p = reinterpret_cast<int4*>(dst);
    p[0] = make_int4(M[0], M[1], M[2], M[3]);
    p[1] = make_int4(M[4], M[5], M[6], M[7]);
    p[2] = make_int4(D[0], D[1], D[2], D[3]);
    p[3] = make_int4(D[4], D[5], D[6], D[7]);
}

__device__ __forceinline__ void load_qc8(const uint8_t* qs, int B, uint8_t* qc8) {
    uint2 w = *reinterpret_cast<const uint2*>(qs + (int64_t)B * BLK);
#pragma unroll
    for (int l = 0; l < 4; l++) {
        qc8[l] = (uint8_t)(w.x >> (8 * l));
        qc8[4 + l] = (uint8_t)(w.y >> (8 * l));
    }
}

__device__ __forceinline__ int64_t align16(int64_t x) { return (x + 15) & ~(int64_t)15; }

struct RowShared {
    int32_t Bs, Be, bn, e0, d, status;
    int64_t st, tb;  // the row's row-store offset and record offset
};

// Summary of one thread's block that lets another thread finalise the block's
// last cell (finalize_last): its exclusive scan prefix without the chunk
// carry, the max of its scan keys of cells 0..6, its H0[7].
struct CellSum {
    int32_t P, k06, h07;
};

// The CTA that fills one alignment. One barrier per chunk: every warp's
// last lane publishes (warp-inclusive key max, its exclusive prefix, k06,
// H0[7]) into a double-buffered array; after the barrier each warp forms the
// cross-warp prefix itself, and lane 0 of every warp has the summary of its
// left neighbour (the previous warp's last lane).
template <int NT>
struct CtaGroup {
    static constexpr int SIZE = NT;
    static constexpr int NW = NT / 32;
    int4* s_sum;  // [2][NW]
    unsigned long long* s_key;
    RowShared* sr;  // [2]: row i's header in sr[i & 1]
    int32_t* upd;   // [UPD_INTS]: the adaptive update's inputs (adaptive band only)
    __device__ __forceinline__ int tid() const { return threadIdx.x; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
    // P: exclusive prefix max of the aggregates (INT_MIN for thread 0), total:
    // the max over the group, left: the summary of the thread to the left
    // (lane 0 of warps >= 1 only), last: the summary of the group's last thread.
    __device__ __forceinline__ void scan(int xp, int32_t agg, int32_t k06, int32_t h07, int32_t& P, int32_t& total,
                                         CellSum& left, CellSum& last) const {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        const int32_t incl = warp_incl_max(agg);
        int32_t ex = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) ex = INT_MIN;
        int4* buf = s_sum + xp * NW;
        if (lane == 31) buf[wid] = make_int4(incl, ex, k06, h07);
        __syncthreads();
        const int32_t wv = warp_incl_max(lane < NW ? buf[lane].x : INT_MIN);  // inclusive over warps
        const int32_t wex1 = __shfl_sync(0xffffffffu, wv, wid >= 1 ? wid - 1 : 0);
        const int32_t wex2 = __shfl_sync(0xffffffffu, wv, wid >= 2 ? wid - 2 : 0);
        const int32_t wlast = __shfl_sync(0xffffffffu, wv, NW >= 2 ? NW - 2 : 0);
        total = __shfl_sync(0xffffffffu, wv, NW - 1);
        P = mx(ex, wid >= 1 ? wex1 : INT_MIN);
        if (wid >= 1) {
            const int4 L = buf[wid - 1];
            left.P = mx(L.y, wid >= 2 ? wex2 : INT_MIN);
            left.k06 = L.z;
            left.h07 = L.w;
        }
        const int4 L = buf[NW - 1];
        last.P = mx(L.y, NW >= 2 ? wlast : INT_MIN);
        last.k06 = L.z;
        last.h07 = L.w;
    }
    __device__ __forceinline__ unsigned long long max_u64(unsigned long long v) const {
        v = warp_max_u64(v);
        if ((threadIdx.x & 31) == 0) s_key[threadIdx.x >> 5] = v;
        __syncthreads();
        unsigned long long k = 0ull;
        for (int w = 0; w < NW; w++) k = s_key[w] > k ? s_key[w] : k;
        return k;
    }
};

// M and I of the last cell of the block summarised by `sm` (block index b),
// given the chunk carry: row 0 has M = H0 and I = NEG_INF.
__device__ __forceinline__ void summary_last(const Scoring& sc, int row, int b, const CellSum& sm, bool haveP,
                                             int32_t carryP, int32_t& M7, int32_t& I7) {
    if (row == 0) {
        M7 = sm.h07;
        I7 = NEG_INF;
        return;
    }
    const int32_t P = haveP ? mx(sm.P, carryP) : sm.P;
    finalize_last(sc, b * BLK, P, sm.k06, sm.h07, M7, I7);
}

// adaptive_update (dp_rowops.h, src/align.cpp:1516-1568) with the warp: the
// predecessors' slope test and the successors' band updates run one lane per
// edge (successors are distinct rows, so their updates do not collide); lane 0
// settles row i's own state in between. Same results as the serial version.
static __device__ void adaptive_update_warp(const DpArgs& a, int i, int Bs, int max_j, int lane) {
    const int n = a.v.n;
    int32_t* Mp = a.state + AB_MP * n;
    int32_t* Sl = a.state + AB_SL * n;
    int32_t* Pl = a.state + AB_PL * n;
    int32_t* Pr = a.state + AB_PR * n;
    int32_t* Ol = a.state + AB_OL * n;
    int32_t* Or = a.state + AB_OR * n;
    int32_t* Ow = a.state + AB_OW * n;
    const int max_acj = Bs * BLK + max_j;
    const bool base_match = (int)a.v.base[i] == (int)a.qs[max_acj + 1];  // cur.base == seq[max_acj]
    int sl_best = INT_MIN, max_slp = 0;
    bool is_match = false;
    if (base_match) {
        const int e0 = a.v.in_ptr[i], e1 = a.v.in_ptr[i + 1];
        for (int e = e0 + lane; e < e1; e += 32) {
            const int p = a.v.in_row[e];
            const int slp = Sl[p];
            max_slp = max(max_slp, slp);
            if (Mp[p] + 1 == max_acj) {
                is_match = true;
                sl_best = max(sl_best, slp + 1);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            max_slp = max(max_slp, __shfl_xor_sync(0xffffffffu, max_slp, o));
            sl_best = max(sl_best, __shfl_xor_sync(0xffffffffu, sl_best, o));
        }
        is_match = __any_sync(0xffffffffu, is_match);
    }
    int sl_i = 0, ow_i = 0, ol_i = 0, or_i = 0;
    if (lane == 0) {
        Mp[i] = max_acj;
        sl_i = Sl[i];
        ow_i = Ow[i];
        ol_i = Ol[i];
        or_i = Or[i];
        if (is_match) sl_i = mx(sl_i, sl_best);
        if (!is_match && max_slp < 30) ow_i = mn(ow_i + max_slp + 1, 5 * a.w);
        if (sl_i >= 30) {
            ol_i = or_i = max_acj - a.v.hq_loc[i];
            ow_i = 0;
        }
        Sl[i] = sl_i;
        Ow[i] = ow_i;
        Ol[i] = ol_i;
        Or[i] = or_i;
    }
    sl_i = __shfl_sync(0xffffffffu, sl_i, 0);
    ow_i = __shfl_sync(0xffffffffu, ow_i, 0);
    ol_i = __shfl_sync(0xffffffffu, ol_i, 0);
    or_i = __shfl_sync(0xffffffffu, or_i, 0);
    const int o0 = a.v.out_ptr[i], o1 = a.v.out_ptr[i + 1];
    for (int e = o0 + lane; e < o1; e += 32) {
        const int s = a.v.out_row[e];
        if (sl_i >= 30) {
            Ol[s] = ol_i;
            Or[s] = or_i;
        } else {
            Ol[s] = mn(Ol[s], ol_i);
            Or[s] = mx(Or[s], or_i);
        }
        Pl[s] = mn(Pl[s], max_acj);
        Pr[s] = mx(Pr[s], max_acj + 1);
        Ow[s] = ow_i ? mx(Ow[s], ow_i) : ow_i;
    }
    __syncwarp();
}

// prefetched adaptive-update inputs (int32 slots): predecessors' Sl, Mp; successors'
// Ol, Or, Pl, Pr, Ow and row index; the row's own Sl, Ow, Ol, Or
constexpr int UPD_PSL = 0, UPD_PMP = 32, UPD_SOL = 64, UPD_SOR = 96, UPD_SPL = 128, UPD_SPR = 160, UPD_SOW = 192,
              UPD_SROW = 224, UPD_OWN = 256, UPD_INTS = 260, UPD_BYTES = 1088;

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit_all() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// adaptive_update_warp with its inputs already in shared memory (copied with
// cp.async when the row started; nothing else writes them in between: the
// predecessors are finished, and only this row's update changes its own and
// its successors' state). Needs d <= 32 predecessors and ns <= 32 successors.
static __device__ void adaptive_update_pf(const DpArgs& a, int i, int Bs, int max_j, int lane, const int32_t* upd, int d,
                                   int ns, int base_i, int hql, const uint8_t* __restrict__ qf) {
    const int n = a.v.n;
    int32_t* Mp = a.state + AB_MP * n;
    int32_t* Sl = a.state + AB_SL * n;
    int32_t* Pl = a.state + AB_PL * n;
    int32_t* Pr = a.state + AB_PR * n;
    int32_t* Ol = a.state + AB_OL * n;
    int32_t* Or = a.state + AB_OR * n;
    int32_t* Ow = a.state + AB_OW * n;
    const int max_acj = Bs * BLK + max_j;
    const bool base_match = base_i == (int)qf[max_acj + 1];  // cur.base == seq[max_acj]
    int sl_best = INT_MIN, max_slp = 0;
    bool is_match = false;
    if (base_match) {
        if (lane < d) {
            const int slp = upd[UPD_PSL + lane];
            max_slp = slp;
            if (upd[UPD_PMP + lane] + 1 == max_acj) {
                is_match = true;
                sl_best = slp + 1;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            max_slp = max(max_slp, __shfl_xor_sync(0xffffffffu, max_slp, o));
            sl_best = max(sl_best, __shfl_xor_sync(0xffffffffu, sl_best, o));
        }
        is_match = __any_sync(0xffffffffu, is_match);
    }
    int sl_i = upd[UPD_OWN + 0], ow_i = upd[UPD_OWN + 1], ol_i = upd[UPD_OWN + 2], or_i = upd[UPD_OWN + 3];
    if (is_match) sl_i = mx(sl_i, sl_best);
    if (!is_match && max_slp < 30) ow_i = mn(ow_i + max_slp + 1, 5 * a.w);
    if (sl_i >= 30) {
        ol_i = or_i = max_acj - hql;
        ow_i = 0;
    }
    if (lane == 0) {
        Mp[i] = max_acj;
        Sl[i] = sl_i;
        Ow[i] = ow_i;
        Ol[i] = ol_i;
        Or[i] = or_i;
    }
    if (lane < ns) {
        const int s = upd[UPD_SROW + lane];
        Ol[s] = sl_i >= 30 ? ol_i : mn(upd[UPD_SOL + lane], ol_i);
        Or[s] = sl_i >= 30 ? or_i : mx(upd[UPD_SOR + lane], or_i);
        Pl[s] = mn(upd[UPD_SPL + lane], max_acj);
        Pr[s] = mx(upd[UPD_SPR + lane], max_acj + 1);
        Ow[s] = ow_i ? mx(upd[UPD_SOW + lane], ow_i) : ow_i;
    }
    __syncwarp();
}

// Row header of row i (one thread): band, placement in the row store, record
// offset and status; advances the bump offsets st_next / tb_next.
__device__ __forceinline__ void row_header(const DpArgs& a, int i, int m, int64_t& st_next, int64_t& tb_next,
                                           RowShared& sr) {
    int Bs, Be;
    row_band(a, i, m, Bs, Be);
    if (i == 0) Bs = 0;
    const int bn = Be - Bs - 1;
    const int e0 = a.v.in_ptr[i];
    const int d = i == 0 ? 0 : a.v.in_ptr[i + 1] - e0;
    int st = ST_OK;
    const int bpc = d >= 2 ? 4 : 1;
    int64_t row_st = st_next;
    bool linear = true;
    if (a.ring_rows > 0) {
        int maxs = i;
        for (int e = a.v.out_ptr[i]; e < a.v.out_ptr[i + 1]; e++) maxs = max(maxs, a.v.out_row[e]);
        const bool spill = (maxs - i >= a.ring_rows) || (bn > a.ring_blocks);
        if (!spill) {
            row_st = (int64_t)(i % a.ring_rows) * a.ring_blocks * 16;
            linear = false;
        }
    }
    if (bn < 0) st = ST_DEGENERATE;
    else if (d > MAX_MULTI_PRED) st = ST_INDEGREE;
    else if ((linear && row_st + (int64_t)bn * 16 > a.rs_cap) || tb_next + (int64_t)bn * BLK * bpc > a.tb_cap)
        st = ST_OOM;
    if (linear && st == ST_OK) st_next = row_st + (int64_t)bn * 16;
    sr.Bs = Bs; sr.Be = Be; sr.bn = bn; sr.e0 = e0; sr.d = d; sr.status = st;
    sr.st = row_st;
    sr.tb = tb_next;
    if (st == ST_OK) {
        RowMeta rm;
        rm.Bs = Bs; rm.Be = Be; rm.st = row_st; rm.tb = tb_next;
        a.meta[i] = rm;
        tb_next = align16(tb_next + (int64_t)bn * BLK * bpc);
    }
}

// Fill all rows of one alignment with group G (see the file comment). Thread
// 0 prepares row i+1's header right after row i's adaptive update, so one
// barrier ends a row and publishes the next header (double-buffered).
template <class G>
__device__ void dp_fill(const G& g, const DpArgs& a) {
    constexpr int NT = G::SIZE;
    const int tid = g.tid();
    const int n = a.v.n, m = a.qlen + 1;
    const bool adaptive = a.f > 0 && a.ab_band;
    const Scoring sc = a.sc;

    if (adaptive)
        for (int r = tid; r < n; r += NT) adaptive_init_entry(a, r, m);
    g.sync();
    int64_t st_next = a.ring_rows > 0 ? (int64_t)a.ring_rows * a.ring_blocks * 16 : 0, tb_next = 0;  // thread 0
    if (tid == 0) row_header(a, 0, m, st_next, tb_next, g.sr[0]);
    g.sync();

    int64_t cells = 0;
    int xp = 0;  // parity of the group's scan buffer, flips every chunk
    for (int i = 0; i < n; i++) {
        const RowShared& sr = g.sr[i & 1];
        const int Bs = sr.Bs, bn = sr.bn, e0 = sr.e0, d = sr.d;
        const int64_t rst = sr.st, rtb = sr.tb;
        if (sr.status != ST_OK) {
            if (tid == 0) a.out[0] = sr.status;
            return;
        }
        // the adaptive update's inputs, copied by warp 0 while the row is filled
        // (nothing else writes them before the update: the predecessors are done
        // and only this row's update changes its own and its successors' state)
        int ns = 0, base_i = 0, hql = 0;
        bool pf = false;
        if (adaptive && i >= 1 && tid < 32) {
            const int o0 = a.v.out_ptr[i];
            ns = a.v.out_ptr[i + 1] - o0;
            pf = d <= 32 && ns <= 32;
            if (pf) {
                base_i = a.v.base[i];
                hql = a.v.hq_loc[i];
                const int32_t* st_ = a.state;
                if (tid < ns) {
                    const int s = a.v.out_row[o0 + tid];
                    g.upd[UPD_SROW + tid] = s;
                    cp_async4(g.upd + UPD_SOL + tid, st_ + AB_OL * n + s);
                    cp_async4(g.upd + UPD_SOR + tid, st_ + AB_OR * n + s);
                    cp_async4(g.upd + UPD_SPL + tid, st_ + AB_PL * n + s);
                    cp_async4(g.upd + UPD_SPR + tid, st_ + AB_PR * n + s);
                    cp_async4(g.upd + UPD_SOW + tid, st_ + AB_OW * n + s);
                }
                if (tid < 4) {
                    const int arr = tid == 0 ? AB_SL : tid == 1 ? AB_OW : tid == 2 ? AB_OL : AB_OR;
                    cp_async4(g.upd + UPD_OWN + tid, st_ + arr * n + i);
                }
                if (tid < d) {
                    const int p = a.v.in_row[e0 + tid];
                    cp_async4(g.upd + UPD_PSL + tid, st_ + AB_SL * n + p);
                    cp_async4(g.upd + UPD_PMP + tid, st_ + AB_MP * n + p);
                }
                cp_async_commit_all();
            }
        }
        cells += (int64_t)bn * BLK;
        const int nch = (bn + NT - 1) / NT;
        int32_t carryP = 0, carryM = NEG_INF, carryI = NEG_INF;
        bool haveP = false;
        unsigned long long best = 0ull;
        for (int c = 0; c < nch; c++) {
            const int b = c * NT + tid;
            const bool act = b < bn;
            const int B = Bs + b;
            int32_t Mpre[BLK], Dv[BLK], H0[BLK], M[BLK], I[BLK];
            int32_t cMb[BLK], cDb[BLK], cmprev = NEG_INF;
            PredMask cmk;
            cmk.blk_in = cmk.prev_in = cmk.diag = false;
            uint8_t qc8[BLK];
#pragma unroll
            for (int l = 0; l < BLK; l++) {
                Mpre[l] = NEG_INF;
                Dv[l] = NEG_INF;
                cMb[l] = cDb[l] = NEG_INF;
            }
            if (act) {
                load_qc8(a.qs, B, qc8);
                if (i == 0) {
#pragma unroll
                    for (int l = 0; l < BLK; l++) Mpre[l] = (b == 0 && l == 0) ? 0 : NEG_INF;
                }
                for (int e = e0; e < e0 + d; e++) {
                    const int pr = a.v.in_row[e];
                    const RowMeta pm = a.meta[pr];
                    const PredMask mk = pred_mask(B, pm.Bs, pm.Be);
                    const int32_t* src = a.rs + pm.st;
                    int32_t Mb[BLK], Db[BLK];
                    int32_t mprev = NEG_INF;
                    if (mk.prev_in) mprev = src[(int64_t)(B - 1 - pm.Bs) * 16 + 7];
                    if (mk.blk_in) {
                        load_block16(src + (int64_t)(B - pm.Bs) * 16, Mb, Db);
                        pass1_pred(sc, mk, b == 0, a.v.in_base[e], Mb, Db, mprev, qc8, Mpre, Dv);
                    }
                    if (d == 1) {
                        cmk = mk;
                        cmprev = mprev;
                        if (mk.blk_in) {
#pragma unroll
                            for (int l = 0; l < BLK; l++) { cMb[l] = Mb[l]; cDb[l] = Db[l]; }
                        }
                    }
                }
            }
            int32_t k06 = INT_MIN, agg = INT_MIN;
#pragma unroll
            for (int l = 0; l < BLK; l++) {
                H0[l] = mx(Mpre[l], Dv[l]);
                if (act) {
                    const int32_t key = scan_key(H0[l], b * BLK + l, sc.e1);
                    if (l < BLK - 1) k06 = mx(k06, key);
                    agg = mx(agg, key);
                }
            }
            // group exclusive prefix max of the per-thread aggregates
            int32_t chunk_total, P;
            CellSum left, last;
            g.scan(xp, agg, k06, H0[BLK - 1], P, chunk_total, left, last);
            xp ^= 1;
            if (haveP) P = mx(P, carryP);
            if (act) {
                if (i == 0) {
#pragma unroll
                    for (int l = 0; l < BLK; l++) { M[l] = H0[l]; I[l] = NEG_INF; }
                } else {
                    finalize_block(sc, b * BLK, P, H0, M, I);
                }
            } else {
#pragma unroll
                for (int l = 0; l < BLK; l++) { M[l] = NEG_INF; I[l] = NEG_INF; }
            }
            // left neighbour of the block's cell 0: the previous lane, the
            // previous warp's last lane (from its summary), or the chunk carry
            int32_t Ml0 = __shfl_up_sync(0xffffffffu, M[BLK - 1], 1);
            int32_t Il0 = __shfl_up_sync(0xffffffffu, I[BLK - 1], 1);
            if ((tid & 31) == 0) {
                if (tid == 0) {
                    Ml0 = carryM;
                    Il0 = carryI;
                } else {
                    summary_last(sc, i, b - 1, left, haveP, carryP, Ml0, Il0);
                }
            }
            if (c + 1 < nch) summary_last(sc, i, c * NT + NT - 1, last, haveP, carryP, carryM, carryI);
            carryP = haveP ? mx(carryP, chunk_total) : chunk_total;
            haveP = true;
            if (act) {
                FlagAcc acc;
                flag_acc_init(acc);
                if (d == 1) {
                    if (cmk.blk_in || cmk.prev_in)
                        flags_pred(sc, cmk, a.v.in_base[e0], a.v.in_w[e0], 0, cMb, cDb, cmprev, qc8, M, Dv, acc);
                } else {
                    for (int e = e0; e < e0 + d; e++) {
                        const int pr = a.v.in_row[e];
                        const RowMeta pm = a.meta[pr];
                        const PredMask mk = pred_mask(B, pm.Bs, pm.Be);
                        if (!(mk.blk_in || mk.prev_in)) continue;
                        const int32_t* src = a.rs + pm.st;
                        int32_t Mb[BLK], Db[BLK];
                        int32_t mprev = NEG_INF;
                        if (mk.prev_in) mprev = src[(int64_t)(B - 1 - pm.Bs) * 16 + 7];
                        if (mk.blk_in) load_block16(src + (int64_t)(B - pm.Bs) * 16, Mb, Db);
                        else {
#pragma unroll
                            for (int l = 0; l < BLK; l++) Mb[l] = Db[l] = NEG_INF;
                        }
                        flags_pred(sc, mk, a.v.in_base[e], a.v.in_w[e], e - e0, Mb, Db, mprev, qc8, M, Dv, acc);
                    }
                }
                const int ind = a.v.ind[i];
                if (d >= 2) {
                    uint32_t r[BLK];
#pragma unroll
                    for (int l = 0; l < BLK; l++) {
                        const int32_t Ml = l > 0 ? M[l - 1] : Ml0, Il = l > 0 ? I[l - 1] : Il0;
                        r[l] = encode_wide(own_flags(sc, b * BLK + l, M[l], Dv[l], I[l], Ml, Il), acc, l, ind);
                    }
                    uint4* dst = reinterpret_cast<uint4*>(a.tb + rtb + (int64_t)b * BLK * 4);
                    dst[0] = make_uint4(r[0], r[1], r[2], r[3]);
                    dst[1] = make_uint4(r[4], r[5], r[6], r[7]);
                } else {
                    uint32_t lo = 0, hi = 0;
#pragma unroll
                    for (int l = 0; l < BLK; l++) {
                        const int32_t Ml = l > 0 ? M[l - 1] : Ml0, Il = l > 0 ? I[l - 1] : Il0;
                        uint32_t v = encode_small(own_flags(sc, b * BLK + l, M[l], Dv[l], I[l], Ml, Il), acc, l, ind);
                        if (l < 4) lo |= v << (8 * l);
                        else hi |= v << (8 * (l - 4));
                    }
                    *reinterpret_cast<uint2*>(a.tb + rtb + (int64_t)b * BLK) = make_uint2(lo, hi);
                }
                store_block16(a.rs + rst + (int64_t)b * 16, M, Dv);
                if (adaptive) {
#pragma unroll
                    for (int l = 0; l < BLK; l++) {
                        unsigned long long key = ((unsigned long long)((uint32_t)M[l] ^ 0x80000000u) << 32) |
                                                 (unsigned long long)(0xffffffffu - (uint32_t)(b * BLK + l));
                        best = key > best ? key : best;
                    }
                }
            }
        }
        if (adaptive && i >= 1) {
            const unsigned long long k = g.max_u64(best);
            if (tid < 32) {
                const int max_j = bn > 0 ? (int)(0xffffffffu - (uint32_t)(k & 0xffffffffu)) : 0;
                if (pf) {
                    cp_async_wait_all();
                    __syncwarp();
                    adaptive_update_pf(a, i, Bs, max_j, tid, g.upd, d, ns, base_i, hql, a.qs);
                } else {
                    adaptive_update_warp(a, i, Bs, max_j, tid);
                }
            }
        }
        if (tid == 0 && i + 1 < n) row_header(a, i + 1, m, st_next, tb_next, g.sr[(i + 1) & 1]);
        g.sync();
    }
    if (tid == 0) {
        const RowMeta last = a.meta[n - 1];
        const int jm = m - last.Bs * BLK;
        // column m lies in the last row's band (tlen[end] - tlen[end] = 0); the
        // guard only keeps a malformed window from reading outside its row
        const bool inb = jm >= 0 && jm / BLK < last.Be - last.Bs - 1;
        a.out[1] = inb ? a.rs[last.st + (int64_t)(jm / BLK) * 16 + jm % BLK] : NEG_INF;
        a.out[3] = (int32_t)(cells > INT_MAX ? INT_MAX : cells);
        a.out[0] = ST_OK;
    }
}

// Backtrack by one warp: all 32 lanes call it with the same arguments and
// take the same steps as backtrack_records (dp_rowops.h, src/align.cpp:
// 1572-1736), with the same results; lane 0 writes the moves. What differs is
// how the data arrive: the lanes fetch ahead along the diagonal, lane k
// loading the row header, record, query code and first predecessor edge of
// cell (i0 - k, acj0 - k), so a run of diagonal moves to the previous row
// costs no further memory round trip. Any other move starts a new fetch at
// the cell it reaches.
static __device__ __noinline__ int32_t backtrack_warp(const DpArgs& a, int m, int lane, int32_t& nmoves) {
    int i = a.v.n - 1, acj = m, op = ALL_OP;
    int32_t nm = 0;
    int i0 = -1, a0 = 0;  // origin of the fetched diagonal
    int f_Bs = 0, f_Be = 0, f_e0 = 0, f_d = 0, f_qc = 4, f_row0 = 0, f_base0 = 0;
    uint32_t f_rec = 0;
    while (i > 0 || acj > 0) {
        int k = i0 - i;
        if (!(i0 >= 0 && k >= 0 && k < 32 && a0 - acj == k)) {
            i0 = i;
            a0 = acj;
            k = 0;
            const int r = i0 - lane, c = a0 - lane;
            f_Bs = f_Be = f_e0 = f_d = f_row0 = f_base0 = 0;
            f_qc = 4;
            f_rec = 0;
            if (r >= 0 && c >= 0) {
                const RowMeta rm = a.meta[r];
                f_Bs = rm.Bs;
                f_Be = rm.Be;
                f_e0 = a.v.in_ptr[r];
                f_d = a.v.in_ptr[r + 1] - f_e0;
                f_qc = c > 0 ? a.qs[c] : 4;
                const int j = c - rm.Bs * BLK, bn = rm.Be - rm.Bs - 1;
                if (c <= (rm.Be - 1) * BLK && c >= rm.Bs * BLK && j < bn * BLK)
                    f_rec = f_d >= 2 ? *reinterpret_cast<const uint32_t*>(a.tb + rm.tb + (int64_t)j * 4)
                                     : (uint32_t)a.tb[rm.tb + j];
                if (f_d >= 1) {
                    f_row0 = a.v.in_row[f_e0];
                    f_base0 = a.v.in_base[f_e0];
                }
            }
        }
        const int Bs = __shfl_sync(0xffffffffu, f_Bs, k), Be = __shfl_sync(0xffffffffu, f_Be, k);
        const int e0 = __shfl_sync(0xffffffffu, f_e0, k), d = __shfl_sync(0xffffffffu, f_d, k);
        const int qck = __shfl_sync(0xffffffffu, f_qc, k);
        const int row0 = __shfl_sync(0xffffffffu, f_row0, k), base0 = __shfl_sync(0xffffffffu, f_base0, k);
        const uint32_t raw = __shfl_sync(0xffffffffu, f_rec, k);
        if (acj > (Be - 1) * BLK || acj < Bs * BLK) { nmoves = nm; return ST_BAND_ESCAPE; }
        const int j = acj - Bs * BLK;
        const int bn = Be - Bs - 1;
        if (j >= bn * BLK) { nmoves = nm; return ST_BT_FAIL; }
        const Rec r = d >= 2 ? decode_wide(raw) : decode_small((uint8_t)raw);
        if (nm + 1 > a.moves_cap) { nmoves = nm; return ST_OOM; }
        const int qc = acj > 0 ? qck : 4;
        if ((op & M_OP) && acj > 0 && r.m1 >= 0) {
            const bool first = r.m1 == 0 && d >= 1;
            const int p = first ? row0 : a.v.in_row[e0 + r.m1];
            const int pb = first ? base0 : (int)a.v.in_base[e0 + r.m1];
            if (lane == 0) a.moves[nm] = mv_pack(pb == qc ? MV_MATCH : MV_MISMATCH, p, qc);
            nm++;
            op = ALL_OP; i = p; acj--;
            continue;
        }
        if ((op & D_OP) && (op == D_OP || r.eqMD) && r.dpos >= 0) {
            i = r.dpos == 0 && d >= 1 ? row0 : a.v.in_row[e0 + r.dpos];
            op = r.dext ? D_OP : (M_OP | I_OP);
            continue;
        }
        if ((op & I_OP) && acj > 0 && j >= 1 && (op == I_OP || r.eqMI)) {
            if (r.iopen) {
                if (lane == 0) a.moves[nm] = mv_pack(MV_INSERT, 0, qc);
                nm++;
                op = M_OP | D_OP; acj--;
                continue;
            }
            if (r.iext) {
                if (lane == 0) a.moves[nm] = mv_pack(MV_INSERT, 0, qc);
                nm++;
                op = I_OP; acj--;
                continue;
            }
        }
        if ((op & M_OP) && acj > 0 && r.m4 >= 0) {
            const bool first = r.m4 == 0 && d >= 1;
            const int p = first ? row0 : a.v.in_row[e0 + r.m4];
            const int pb = first ? base0 : (int)a.v.in_base[e0 + r.m4];
            if (lane == 0) a.moves[nm] = mv_pack(pb == qc ? MV_MATCH : MV_MISMATCH, p, qc);
            nm++;
            op = ALL_OP; i = p; acj--;
            continue;
        }
        nmoves = nm;
        return ST_BT_FAIL;
    }
    nmoves = nm;
    return ST_OK;
}

// one CTA per job: fill every row, then warp 0 backtracks
template <int NT>
__global__ void __launch_bounds__(NT, 1) k_plain(const DpArgs* __restrict__ jobs) {
    __shared__ DpArgs sa;
    if (threadIdx.x == 0) sa = jobs[blockIdx.x];
    __syncthreads();
    const DpArgs& a = sa;
    if (a.v.n <= 0) {
        if (threadIdx.x == 0) a.out[0] = ST_BAD_ARG;
        return;
    }
    constexpr int NW = NT / 32;
    __shared__ int4 s_sum[2 * NW];
    __shared__ unsigned long long s_key[NW];
    __shared__ RowShared sr[2];
    __shared__ int32_t s_upd[UPD_INTS];
    CtaGroup<NT> g{s_sum, s_key, sr, s_upd};
    dp_fill(g, a);
    __syncthreads();
    if (threadIdx.x < 32 && a.out[0] == ST_OK) {
        int32_t nm = 0;
        const int32_t st = backtrack_warp(a, a.qlen + 1, threadIdx.x, nm);
        if (threadIdx.x == 0) {
            a.out[0] = st;
            a.out[2] = nm;
        }
    }
}

}  // namespace pb
