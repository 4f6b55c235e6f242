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
//      H0[k] - k*e1 (warp shuffles + one shared-memory level).
//   3. final M and I, the backtrack records of the block (own-row tests plus
//      one comparison sweep over the predecessors), and the row's M/D blocks
//      are written back to global memory, all 16-byte vector stores.
//   4. with the adaptive band, a CTA argmax of M, then thread 0 propagates
//      the band state to the successors (src/align.cpp:1516-1568).
// After the last row thread 0 walks the records back from (n-1, m).
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
    int64_t st, tb;
    int64_t st_next, tb_next;  // next free row-store offset (spill area when ringed), next record offset
};

// A thread group that fills one alignment: the whole CTA (plain kernel) ...
template <int NT>
struct CtaGroup {
    static constexpr int SIZE = NT;
    static constexpr int NW = NT / 32;
    int32_t* s_scan;
    int32_t* s_scan2;
    int32_t* s_lastM;
    int32_t* s_lastI;
    unsigned long long* s_key;
    RowShared* sr;
    __device__ __forceinline__ int tid() const { return threadIdx.x; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
    // exclusive prefix max of per-thread aggregates; total = max over the group
    __device__ __forceinline__ int32_t excl_max(int32_t agg, int32_t& total) const {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        const int32_t incl = warp_incl_max(agg);
        int32_t ex_w = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) ex_w = INT_MIN;
        if (lane == 31) s_scan[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            int32_t v = lane < NW ? s_scan[lane] : INT_MIN;
            v = warp_incl_max(v);
            if (lane < NW) s_scan2[lane] = v;
        }
        __syncthreads();
        total = s_scan2[NW - 1];
        return mx(ex_w, wid > 0 ? s_scan2[wid - 1] : INT_MIN);
    }
    // left neighbour (M, I of the previous thread's last cell) and the values
    // of the group's last thread (the carry into the next chunk)
    __device__ __forceinline__ void edges(int32_t m7, int32_t i7, int32_t carryM, int32_t carryI, int32_t& Ml0,
                                          int32_t& Il0, int32_t& nextM, int32_t& nextI) const {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        const int32_t upM = __shfl_up_sync(0xffffffffu, m7, 1);
        const int32_t upI = __shfl_up_sync(0xffffffffu, i7, 1);
        if (lane == 31) { s_lastM[wid] = m7; s_lastI[wid] = i7; }
        __syncthreads();
        Ml0 = lane > 0 ? upM : (wid > 0 ? s_lastM[wid - 1] : carryM);
        Il0 = lane > 0 ? upI : (wid > 0 ? s_lastI[wid - 1] : carryI);
        nextM = s_lastM[NW - 1];
        nextI = s_lastI[NW - 1];
    }
    __device__ __forceinline__ unsigned long long max_u64(unsigned long long v) const {
        v = warp_max_u64(v);
        if ((threadIdx.x & 31) == 0) s_key[threadIdx.x >> 5] = v;
        __syncthreads();
        unsigned long long k = 0ull;
        for (int w = 0; w < NW; w++) k = s_key[w] > k ? s_key[w] : k;
        return k;
    }
    // thread 0 wrote *sr; make it visible to the group
    __device__ __forceinline__ void publish() const { __syncthreads(); }
};

// ... or one warp (batched kernel: one warp per window)
struct WarpGroup {
    static constexpr int SIZE = 32;
    RowShared* sr;
    __device__ __forceinline__ int tid() const { return threadIdx.x & 31; }
    __device__ __forceinline__ void sync() const { __syncwarp(); }
    __device__ __forceinline__ int32_t excl_max(int32_t agg, int32_t& total) const {
        const int lane = threadIdx.x & 31;
        const int32_t incl = warp_incl_max(agg);
        int32_t ex = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) ex = INT_MIN;
        total = __shfl_sync(0xffffffffu, incl, 31);
        return ex;
    }
    __device__ __forceinline__ void edges(int32_t m7, int32_t i7, int32_t carryM, int32_t carryI, int32_t& Ml0,
                                          int32_t& Il0, int32_t& nextM, int32_t& nextI) const {
        const int lane = threadIdx.x & 31;
        const int32_t upM = __shfl_up_sync(0xffffffffu, m7, 1);
        const int32_t upI = __shfl_up_sync(0xffffffffu, i7, 1);
        Ml0 = lane > 0 ? upM : carryM;
        Il0 = lane > 0 ? upI : carryI;
        nextM = __shfl_sync(0xffffffffu, m7, 31);
        nextI = __shfl_sync(0xffffffffu, i7, 31);
    }
    __device__ __forceinline__ unsigned long long max_u64(unsigned long long v) const { return warp_max_u64(v); }
    __device__ __forceinline__ void publish() const { __syncwarp(); }
};

// Fill all rows of one alignment with group G (see the file comment).
template <class G>
__device__ void dp_fill(const G& g, const DpArgs& a) {
    constexpr int NT = G::SIZE;
    RowShared& sr = *g.sr;
    const int tid = g.tid();
    const int n = a.v.n, m = a.qlen + 1;
    const bool adaptive = a.f > 0 && a.ab_band;
    const Scoring sc = a.sc;

    if (adaptive)
        for (int r = tid; r < n; r += NT) adaptive_init_entry(a, r, m);
    if (tid == 0) {
        sr.st_next = a.ring_rows > 0 ? (int64_t)a.ring_rows * a.ring_blocks * 16 : 0;
        sr.tb_next = 0;
    }
    g.sync();

    int64_t cells = 0;
    for (int i = 0; i < n; i++) {
        if (tid == 0) {
            int Bs, Be;
            row_band(a, i, m, Bs, Be);
            if (i == 0) Bs = 0;
            const int bn = Be - Bs - 1;
            const int e0 = a.v.in_ptr[i];
            const int d = i == 0 ? 0 : a.v.in_ptr[i + 1] - e0;
            int st = ST_OK;
            const int bpc = d >= 2 ? 4 : 1;
            int64_t row_st = sr.st_next;
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
            else if ((linear && row_st + (int64_t)bn * 16 > a.rs_cap) || sr.tb_next + (int64_t)bn * BLK * bpc > a.tb_cap)
                st = ST_OOM;
            if (linear) sr.st_next = row_st + (int64_t)bn * 16;
            sr.Bs = Bs; sr.Be = Be; sr.bn = bn; sr.e0 = e0; sr.d = d; sr.status = st;
            sr.st = row_st;
            sr.tb = sr.tb_next;
            if (st == ST_OK) {
                RowMeta rm;
                rm.Bs = Bs; rm.Be = Be; rm.st = sr.st; rm.tb = sr.tb;
                a.meta[i] = rm;
            }
        }
        g.publish();
        const int Bs = sr.Bs, bn = sr.bn, e0 = sr.e0, d = sr.d;
        const int64_t rst = sr.st, rtb = sr.tb;
        if (sr.status != ST_OK) {
            if (tid == 0) a.out[0] = sr.status;
            return;
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
                    int32_t Mb[BLK], Db[BLK];
                    int32_t mprev = NEG_INF;
                    if (mk.prev_in) mprev = a.rs[pm.st + (int64_t)(B - 1 - pm.Bs) * 16 + 7];
                    if (mk.blk_in) {
                        load_block16(a.rs + pm.st + (int64_t)(B - pm.Bs) * 16, Mb, Db);
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
            int32_t agg = INT_MIN;
#pragma unroll
            for (int l = 0; l < BLK; l++) {
                H0[l] = mx(Mpre[l], Dv[l]);
                if (act) agg = mx(agg, scan_key(H0[l], b * BLK + l, sc.e1));
            }
            // group exclusive prefix max of the per-thread aggregates
            int32_t chunk_total;
            int32_t P = g.excl_max(agg, chunk_total);
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
            // left neighbours of lane 0 of the block
            int32_t Ml0, Il0, nextM, nextI;
            g.edges(M[BLK - 1], I[BLK - 1], carryM, carryI, Ml0, Il0, nextM, nextI);
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
                        int32_t Mb[BLK], Db[BLK];
                        int32_t mprev = NEG_INF;
                        if (mk.prev_in) mprev = a.rs[pm.st + (int64_t)(B - 1 - pm.Bs) * 16 + 7];
                        if (mk.blk_in) load_block16(a.rs + pm.st + (int64_t)(B - pm.Bs) * 16, Mb, Db);
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
            carryP = haveP ? mx(carryP, chunk_total) : chunk_total;
            haveP = true;
            carryM = nextM;
            carryI = nextI;
        }
        if (adaptive && i >= 1) {
            const unsigned long long k = g.max_u64(best);
            if (tid == 0) {
                const int max_j = bn > 0 ? (int)(0xffffffffu - (uint32_t)(k & 0xffffffffu)) : 0;
                adaptive_update(a, i, Bs, max_j);
            }
        }
        if (tid == 0) {
            const int bpc = d >= 2 ? 4 : 1;
            sr.tb_next = align16(rtb + (int64_t)bn * BLK * bpc);
        }
        g.sync();
    }
    if (tid == 0) {
        const RowMeta last = a.meta[n - 1];
        const int jm = m - last.Bs * BLK;
        a.out[1] = a.rs[last.st + (int64_t)(jm / BLK) * 16 + jm % BLK];
        a.out[3] = (int32_t)(cells > INT_MAX ? INT_MAX : cells);
        a.out[0] = ST_OK;
    }
}

// one CTA per job: fill every row, then thread 0 backtracks
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
    __shared__ int32_t s_scan[NW], s_scan2[NW], s_lastM[NW], s_lastI[NW];
    __shared__ unsigned long long s_key[NW];
    __shared__ RowShared sr;
    CtaGroup<NT> g{s_scan, s_scan2, s_lastM, s_lastI, s_key, &sr};
    dp_fill(g, a);
    __syncthreads();
    if (threadIdx.x == 0 && a.out[0] == ST_OK) {
        int32_t nm = 0;
        a.out[0] = backtrack_records(a, a.qlen + 1, nm);
        a.out[2] = nm;
    }
}

}  // namespace pb
