// plain_static.cuh - the single-alignment DP kernel for the static band
// (src/align.cpp:1382-1390; every poa() call without -B/-S): one CTA per
// poa() call, integer-only.
//
// A static row's band, row-store location and record offset depend only on
// hlen/tlen, so they are computed for all rows up front, in parallel
// (prefix sums over the rows), instead of by one thread at the start of every
// row. The fill then needs two CTA barriers per row chunk:
//   1. after pass 1, every warp's last lane publishes a summary of its block
//      (warp-inclusive scan key, its own exclusive prefix, the max of its keys
//      of cells 0..6, its H0[7]); after the barrier each warp derives the
//      cross-warp prefix itself, and lane 0 of every warp derives its left
//      neighbour's final M/I from the summary (finalize_last) — no further
//      exchange is needed for the records;
//   2. at the end of the row, so that its M/D blocks are visible to the next
//      row.
// Recent rows' M/D blocks live in a shared-memory ring (row i in slot
// i % ring_rows); a row with an in-window successor ring_rows or more rows
// ahead, or wider than the ring, goes to the global row store instead. A ring
// row's RowMeta.st holds ~(its offset in the ring), a global row's st >= 0.
// Results are identical to k_plain's: same per-block functions, same records,
// and the same warp backtrack (backtrack_warp).
#pragma once
#include "plain.cuh"

namespace pb {

__device__ __forceinline__ const int32_t* row_src(const int32_t* ring, const int32_t* rs, int64_t st) {
    return st < 0 ? ring + (~st) : rs + st;
}

// CTA-wide exclusive prefix sum (NT threads); total = the sum over the CTA.
template <int NT>
__device__ __forceinline__ int64_t cta_excl_sum(int64_t v, int64_t* s_part, int64_t& total) {
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_part[wid] = x;
    __syncthreads();
    int64_t before = 0;
    total = 0;
#pragma unroll
    for (int k = 0; k < NW; k++) {
        const int64_t p = s_part[k];
        if (k < wid) before += p;
        total += p;
    }
    __syncthreads();  // s_part is reused by the next call
    return before + x - v;
}

template <int NT>
__global__ void __launch_bounds__(NT, 1) k_plain_static(const DpArgs* __restrict__ jobs) {
    constexpr int NW = NT / 32;
    __shared__ DpArgs sa;
    __shared__ int64_t s_part[NW];
    __shared__ int4 s_sum[2 * NW];
    __shared__ unsigned long long s_fail;
    extern __shared__ int4 s_dyn[];
    int32_t* ring = reinterpret_cast<int32_t*>(s_dyn);
    if (threadIdx.x == 0) {
        sa = jobs[blockIdx.x];
        s_fail = ~0ull;
    }
    __syncthreads();
    const DpArgs& a = sa;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int n = a.v.n, m = a.qlen + 1;
    if (n <= 0) {
        if (tid == 0) a.out[0] = ST_BAD_ARG;
        return;
    }
    const int R = a.ring_rows, RB = a.ring_blocks;
    const Scoring sc = a.sc;
    const CtaGroup<NT> g{s_sum, nullptr, nullptr, nullptr};  // scan only

    // ---- rows: band, placement, record offset (src/align.cpp:1382-1391) ----
    int64_t st_run = 0, tb_run = 0;
    for (int r0 = 0; r0 < n; r0 += NT) {
        const int i = r0 + tid;
        int Bs = 0, Be = 1, d = 0;
        bool spill = true;
        if (i < n) {
            band_static(a.f, a.v.hq[i], a.v.tq[i], m, a.w, Bs, Be);
            if (i == 0) Bs = 0;
            d = i == 0 ? 0 : a.v.in_ptr[i + 1] - a.v.in_ptr[i];
            if (R > 0 && Be - Bs - 1 <= RB) {
                int maxs = i;
                for (int e = a.v.out_ptr[i]; e < a.v.out_ptr[i + 1]; e++) maxs = max(maxs, a.v.out_row[e]);
                spill = maxs - i >= R;
            }
        }
        const int bn = Be - Bs - 1;
        const int bnc = bn > 0 ? bn : 0;
        const int bpc = d >= 2 ? 4 : 1;
        int64_t st_tot, tb_tot;
        const int64_t st_off = st_run + cta_excl_sum<NT>(i < n && spill ? (int64_t)bnc * 16 : 0, s_part, st_tot);
        const int64_t tb_off =
            tb_run + cta_excl_sum<NT>(i < n ? align16((int64_t)bnc * BLK * bpc) : 0, s_part, tb_tot);
        st_run += st_tot;
        tb_run += tb_tot;
        if (i < n) {
            int st = ST_OK;
            if (bn < 0) st = ST_DEGENERATE;
            else if (d > MAX_MULTI_PRED) st = ST_INDEGREE;
            else if ((spill && st_off + (int64_t)bn * 16 > a.rs_cap) || tb_off + (int64_t)bn * BLK * bpc > a.tb_cap)
                st = ST_OOM;
            if (st != ST_OK) atomicMin(&s_fail, ((unsigned long long)i << 8) | (unsigned long long)st);
            RowMeta rm;
            rm.Bs = Bs;
            rm.Be = Be;
            rm.st = spill ? st_off : ~((int64_t)(i % R) * RB * 16);
            rm.tb = tb_off;
            a.meta[i] = rm;
        }
    }
    __syncthreads();
    if (s_fail != ~0ull) {  // the first failing row decides the status, as in the row-by-row fill
        if (tid == 0) {
            a.out[0] = (int32_t)(s_fail & 255ull);
            a.out[1] = 0;
            a.out[2] = 0;
            a.out[3] = 0;
        }
        return;
    }

    // ---- fill ----
    int64_t cells = 0;
    int xp = 0;  // parity of s_sum, flips every chunk
    RowMeta nxt = a.meta[0], prevm = nxt;
    int nx_e0 = a.v.in_ptr[0], nx_e1 = a.v.in_ptr[1];
    for (int i = 0; i < n; i++) {
        const RowMeta cur = nxt;
        const int e0 = nx_e0, d = i == 0 ? 0 : nx_e1 - nx_e0;
        if (i + 1 < n) {  // the next row's header, loaded while this row computes
            nxt = a.meta[i + 1];
            nx_e0 = nx_e1;
            nx_e1 = a.v.in_ptr[i + 2];
        }
        const int Bs = cur.Bs, bn = cur.Be - cur.Bs - 1;
        int32_t* dst_rs = cur.st < 0 ? ring + (~cur.st) : a.rs + cur.st;
        uint8_t* dst_tb = a.tb + cur.tb;
        const int ind = a.v.ind[i];
        cells += (int64_t)bn * BLK;
        const int nch = (bn + NT - 1) / NT;
        int32_t carryP = 0, carryM = NEG_INF, carryI = NEG_INF;
        bool haveP = false;
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
                    const RowMeta pm = pr == i - 1 ? prevm : a.meta[pr];
                    const PredMask mk = pred_mask(B, pm.Bs, pm.Be);
                    const int32_t* src = row_src(ring, a.rs, pm.st);
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
            // barrier 1: warp summaries
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
            // left neighbour of the block's cell 0
            int32_t Ml0 = __shfl_up_sync(0xffffffffu, M[BLK - 1], 1);
            int32_t Il0 = __shfl_up_sync(0xffffffffu, I[BLK - 1], 1);
            if (lane == 0) {
                if (wid == 0) {
                    Ml0 = carryM;
                    Il0 = carryI;
                } else {
                    summary_last(sc, i, b - 1, left, haveP, carryP, Ml0, Il0);
                }
            }
            // the chunk's last cell, left neighbour of the next chunk
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
                        const RowMeta pm = pr == i - 1 ? prevm : a.meta[pr];
                        const PredMask mk = pred_mask(B, pm.Bs, pm.Be);
                        if (!(mk.blk_in || mk.prev_in)) continue;
                        const int32_t* src = row_src(ring, a.rs, pm.st);
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
                if (d >= 2) {
                    uint32_t r[BLK];
#pragma unroll
                    for (int l = 0; l < BLK; l++) {
                        const int32_t Ml = l > 0 ? M[l - 1] : Ml0, Il = l > 0 ? I[l - 1] : Il0;
                        r[l] = encode_wide(own_flags(sc, b * BLK + l, M[l], Dv[l], I[l], Ml, Il), acc, l, ind);
                    }
                    uint4* dst = reinterpret_cast<uint4*>(dst_tb + (int64_t)b * BLK * 4);
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
                    *reinterpret_cast<uint2*>(dst_tb + (int64_t)b * BLK) = make_uint2(lo, hi);
                }
                store_block16(dst_rs + (int64_t)b * 16, M, Dv);
            }
        }
        prevm = cur;
        __syncthreads();  // barrier 2: the row's M/D before the next row reads them
    }
    if (tid < 32) {  // warp 0: score, then the backtrack
        int32_t nm = 0;
        const int32_t st = backtrack_warp(a, m, tid, nm);
        if (tid == 0) {
            const RowMeta last = prevm;
            const int jm = m - last.Bs * BLK;
            // column m lies in the last row's band (tlen[end] - tlen[end] = 0); the
            // guard only keeps a malformed window from reading outside its row
            const bool inb = jm >= 0 && jm / BLK < last.Be - last.Bs - 1;
            a.out[1] = inb ? row_src(ring, a.rs, last.st)[(int64_t)(jm / BLK) * 16 + jm % BLK] : NEG_INF;
            a.out[3] = (int32_t)(cells > INT_MAX ? INT_MAX : cells);
            a.out[0] = st;
            a.out[2] = nm;
        }
    }
}

}  // namespace pb
