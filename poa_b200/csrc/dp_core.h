// dp_core.h - per-block arithmetic of the banded POA DP, shared by the sm_100a
// kernels (plain.cu, batch.cu) and, compiled as host C++, by the CPU model the
// tests use to validate this formulation against the oracle.
//
// Formulation (bit-exact with minipoa's poa(), src/align.cpp:1353-1737):
//  * A row is the band of one rank; column blocks of 8 cells (the reference's
//    AVX2 lane count, src/align.cpp:13-19) map to one thread each. Row i
//    covers absolute blocks [Bs, Be); blocks [Bs, Be-1) are computed and block
//    Be-1 is the NEG_INF pad (src/align.cpp:1391, 1446, 1505-1506).
//  * M/D from predecessors (src/align.cpp:1449-1498) keep the reference's
//    block-granular masks: the diagonal from p applies to block B iff
//    max(0,B-1) >= Bs_p && B <= Be_p-2, the vertical iff Bs_p <= B < Be_p-1,
//    and lane 0 of the row's first block reads NEG_INF instead of M_p.
//  * The horizontal recurrence I[j] = max(I[j-1]+e1, M[j-1]+o1),
//    M[j] = max(H0[j], I[j]) (src/align.cpp:1507-1514) is evaluated as a
//    prefix max: because o1 <= e1,
//        I[j] = max(NEG_INF + j*e1, o1 + (j-1)*e1 + max_{k<j}(H0[k] - k*e1)),
//    exact in int32 while |scores| stay far from 2^31 (true for any band
//    narrower than ~10^7 cells).
//  * The backtrack (src/align.cpp:1572-1736) compares raw M/D/I values of the
//    cell, its left neighbour and its predecessors. The fill evaluates every
//    one of those comparisons once, when the values are in registers, and
//    stores the outcome as a compact record per cell: 1 byte for rows with at
//    most one in-window predecessor, 4 bytes (with predecessor indices) for
//    the rest. The backtrack then only reads records.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define PB_HD __host__ __device__ __forceinline__
#define PB_UNROLL _Pragma("unroll")
#else
#define PB_HD inline
#define PB_UNROLL
#endif

namespace pb {

constexpr int BLK = 8;
constexpr int32_t NEG_INF = (int32_t)0xc0c0c0c0;  // src/align.cpp:22
enum { M_OP = 1, D_OP = 2, I_OP = 4, ALL_OP = 7 };  // src/align.cpp:23

// status codes shared with include/poa_b200.h
enum Status : int32_t {
    ST_OK = 0,
    ST_BAND_ESCAPE = 1,   // reference: prints the band and exit(0)s, src/align.cpp:1584-1588
    ST_BT_FAIL = 2,       // reference: " backtrack error", exit(1), src/align.cpp:1730-1731
    ST_BAD_ARG = 3,
    ST_OOM = 4,           // device arena too small for this alignment (host grows it and retries)
    ST_INDEGREE = 5,      // more in-window predecessors than the 4-byte record can index
    ST_DEGENERATE = 6,    // a band with Be-Bs < 1: the reference writes outside its row there
    ST_CAPACITY = 7,      // a batched window outgrew its device graph capacity
    ST_UNSUPPORTED = 9,   // an option outside the path (-p)
};

// record layout -------------------------------------------------------------
// 1-byte record (rows with <= 1 in-window predecessor)
constexpr uint32_t R_EQMD = 1u << 0;   // M == D at this cell
constexpr uint32_t R_EQMI = 1u << 1;   // M == I
constexpr uint32_t R_IOPEN = 1u << 2;  // I == M[j-1] + o1
constexpr uint32_t R_IEXT = 1u << 3;   // I == I[j-1] + e1
constexpr uint32_t R_M1 = 1u << 4;     // match move accepted by the in_weight >= ind/10 rule
constexpr uint32_t R_M4 = 1u << 5;     // any diagonal move
constexpr uint32_t R_DOPEN = 1u << 6;  // D == M_p + o1
constexpr uint32_t R_DEXT = 1u << 7;   // D == D_p + e1 (only when no open)
// 4-byte record (rows with >= 2 in-window predecessors): bits 0..3 as above,
// bit 4 = D move is an extension, then three 9-bit predecessor positions
// (index into the row's in-window predecessor list; 511 = none).
constexpr uint32_t W_DEXT = 1u << 4;
constexpr int W_M1_SHIFT = 5, W_M4_SHIFT = 14, W_D_SHIFT = 23;
constexpr uint32_t W_NONE = 511u;
constexpr int MAX_MULTI_PRED = 510;

struct Scoring {
    int32_t match, mismatch, o1, e1;  // o1 = gap_open1 + gap_ext1, src/align.cpp:1369
};

// per-row bookkeeping written by the fill, read by successors and the backtrack
struct RowMeta {
    int32_t Bs, Be;  // block range [Bs, Be); Be-1 is the pad
    int64_t st;      // offset (int32 units) of this row's M/D blocks in the row store
    int64_t tb;      // byte offset of this row's records
};

PB_HD int32_t add32(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
PB_HD int32_t mx(int32_t a, int32_t b) { return a > b ? a : b; }
PB_HD int32_t mn(int32_t a, int32_t b) { return a < b ? a : b; }

PB_HD int32_t sub_score(const Scoring& s, int pb, int qc) { return pb == qc ? s.match : s.mismatch; }

// Static band of a row, src/align.cpp:1382-1390. h = hlen[aci]-hlen[beg],
// tq = tlen[aci]-tlen[end]; f == 0 means the full band [0, m].
PB_HD void band_static(int f, int h, int tq, int m, int w, int& Bs, int& Be) {
    int Ms, Me;
    if (f > 0) {
        int t = m - tq;
        Ms = mx(0, mn(h, t) - w);
        Me = mn(m, mx(h, t) + w);
    } else {
        Ms = 0;
        Me = m;
    }
    Bs = Ms / BLK;
    Be = Me / BLK + 2;
}

// Adaptive band of a row, src/align.cpp:1433-1444 (and :1410-1414 for row 0).
PB_HD void band_adaptive(int h, int tq, int m, int w, int Pl, int Pr, int Ol, int Or, int Ow,
                         int& Bs, int& Be) {
    int t = m - tq;
    int Ms = mx(0, mn(mn(Pl, h + Ol), t) - w - Ow);
    int Me = mn(m, mx(mx(Pr, h + Or), t) + w + Ow);
    Bs = Ms / BLK;
    Be = Me / BLK + 2;
}

// Predecessor block availability for absolute block B of the current row.
struct PredMask {
    bool blk_in;   // block B computed in p: Bs_p <= B <= Be_p-2  (vertical mask)
    bool prev_in;  // block B-1 computed in p                       (lane-0 diagonal source)
    bool diag;     // the reference's diagonal mask, src/align.cpp:1467
};
PB_HD PredMask pred_mask(int B, int Bs_p, int Be_p) {
    PredMask r;
    r.blk_in = (Bs_p <= B) && (B <= Be_p - 2);
    r.prev_in = (B - 1 >= Bs_p) && (B - 1 <= Be_p - 2);
    r.diag = !((mx(0, B - 1) < Bs_p) || (B > Be_p - 2));
    return r;
}

// Pass 1 of one 8-cell block for one predecessor: diagonal into Mpre, vertical
// into Dv. Mb/Db: p's M/D at this absolute block; mprev: p's M at the cell left
// of the block (valid iff prev_in). first_block: this block is the row's first
// computed block (lane-0 quirk). qc8: query code seq[acj-1] for the 8 cells.
PB_HD void pass1_pred(const Scoring& s, const PredMask& pm, bool first_block, int pbase,
                      const int32_t* Mb, const int32_t* Db, int32_t mprev, const uint8_t* qc8,
                      int32_t* Mpre, int32_t* Dv) {
    if (pm.blk_in) {
PB_UNROLL
        for (int l = 0; l < BLK; l++) {
            Dv[l] = mx(Dv[l], add32(Db[l], s.e1));
            Dv[l] = mx(Dv[l], add32(Mb[l], s.o1));
        }
        if (pm.diag) {
            int32_t d0 = first_block ? NEG_INF : mprev;
            Mpre[0] = mx(Mpre[0], add32(d0, sub_score(s, pbase, qc8[0])));
PB_UNROLL
            for (int l = 1; l < BLK; l++) Mpre[l] = mx(Mpre[l], add32(Mb[l - 1], sub_score(s, pbase, qc8[l])));
        }
    }
}

// A[k] = H0[k] - k*e1 for the prefix-max form of the I recurrence.
PB_HD int32_t scan_key(int32_t h0, int j, int32_t e1) { return add32(h0, -(int32_t)((int64_t)j * e1)); }

// I at column j >= 1 from the prefix max `run` of the scan keys of the cells
// left of j.
PB_HD int32_t i_at(const Scoring& s, int j, int32_t run) {
    int32_t ext = add32(NEG_INF, (int32_t)((int64_t)j * s.e1));
    int32_t opn = add32(add32(s.o1, (int32_t)((int64_t)(j - 1) * s.e1)), run);
    return mx(ext, opn);
}

// Finalise M and I of one block given H0 and the exclusive prefix max P of the
// scan keys of all cells left of the block (ignored when the block holds j=0).
PB_HD void finalize_block(const Scoring& s, int j0, int32_t P, const int32_t* H0, int32_t* M, int32_t* I) {
    int32_t run = P;
    bool have = j0 > 0;
PB_UNROLL
    for (int l = 0; l < BLK; l++) {
        int j = j0 + l;
        int32_t Ij = j == 0 ? NEG_INF : i_at(s, j, run);
        I[l] = Ij;
        M[l] = mx(H0[l], Ij);
        int32_t key = scan_key(H0[l], j, s.e1);
        run = have ? mx(run, key) : key;
        have = true;
    }
}

// M and I of the last cell of a block (j0 + 7) without the block's other
// cells: P as for finalize_block, k06 = max of the scan keys of its cells
// 0..6, h07 = its H0[7]. Equal to finalize_block's M[7], I[7].
PB_HD void finalize_last(const Scoring& s, int j0, int32_t P, int32_t k06, int32_t h07, int32_t& M7, int32_t& I7) {
    const int32_t run = j0 > 0 ? mx(P, k06) : k06;
    I7 = i_at(s, j0 + BLK - 1, run);
    M7 = mx(h07, I7);
}

// Per-cell best-so-far keys for multi-predecessor records: (weight << 10) |
// (1023 - position) so that a larger key = larger in_weight, first on ties.
PB_HD int32_t wkey(int w, int pos) { return (w << 10) | (1023 - pos); }
PB_HD int key_pos(int32_t key) { return 1023 - (key & 1023); }
PB_HD int key_w(int32_t key) { return key >> 10; }

struct FlagAcc {
    int32_t k1[BLK], k4[BLK], kdo[BLK], kde[BLK];  // -1 = none
};
PB_HD void flag_acc_init(FlagAcc& a) {
PB_UNROLL
    for (int l = 0; l < BLK; l++) a.k1[l] = a.k4[l] = a.kdo[l] = a.kde[l] = -1;
}

// Backtrack comparisons against one predecessor (src/align.cpp:1592-1604,
// 1632-1658, 1692-1711) for the 8 cells of a block. acj0 = absolute column of
// lane 0. qc8 = seq[acj-1] per lane.
PB_HD void flags_pred(const Scoring& s, const PredMask& pm, int pbase, int w, int pos,
                      const int32_t* Mb, const int32_t* Db, int32_t mprev, const uint8_t* qc8,
                      const int32_t* M, const int32_t* D, FlagAcc& a) {
    int32_t key = wkey(w, pos);
PB_UNROLL
    for (int l = 0; l < BLK; l++) {
        bool inr = (l == 0) ? pm.prev_in : pm.blk_in;
        if (inr) {
            int32_t mv = (l == 0) ? mprev : Mb[l - 1];
            bool bm = pbase == qc8[l];
            if (M[l] == add32(mv, bm ? s.match : s.mismatch)) {
                if (key > a.k4[l]) a.k4[l] = key;
                if (bm && key > a.k1[l]) a.k1[l] = key;
            }
        }
        if (pm.blk_in) {
            if (D[l] == add32(Mb[l], s.o1) && key > a.kdo[l]) a.kdo[l] = key;
            if (D[l] == add32(Db[l], s.e1) && key > a.kde[l]) a.kde[l] = key;
        }
    }
}

// Own-row flags of one block (I and the M==D / M==I tests).
PB_HD uint32_t own_flags(const Scoring& s, int j, int32_t M, int32_t D, int32_t I, int32_t Mleft, int32_t Ileft) {
    uint32_t r = 0;
    if (M == D) r |= R_EQMD;
    if (M == I) r |= R_EQMI;
    if (j >= 1) {
        if (I == add32(Mleft, s.o1)) r |= R_IOPEN;
        if (I == add32(Ileft, s.e1)) r |= R_IEXT;
    }
    return r;
}

// Encode the 1-byte record of a row with <= 1 in-window predecessor.
PB_HD uint8_t encode_small(uint32_t own, const FlagAcc& a, int l, int ind) {
    uint32_t r = own;
    if (a.k1[l] >= 0 && key_w(a.k1[l]) >= ind / 10) r |= R_M1;
    if (a.k4[l] >= 0) r |= R_M4;
    if (a.kdo[l] >= 0) r |= R_DOPEN;
    else if (a.kde[l] >= 0) r |= R_DEXT;
    return (uint8_t)r;
}

// Encode the 4-byte record of a multi-predecessor row.
PB_HD uint32_t encode_wide(uint32_t own, const FlagAcc& a, int l, int ind) {
    uint32_t r = own & 15u;
    uint32_t m1 = W_NONE, m4 = W_NONE, dd = W_NONE;
    if (a.k1[l] >= 0 && key_w(a.k1[l]) >= ind / 10) m1 = (uint32_t)key_pos(a.k1[l]);
    if (a.k4[l] >= 0) m4 = (uint32_t)key_pos(a.k4[l]);
    if (a.kdo[l] >= 0) dd = (uint32_t)key_pos(a.kdo[l]);
    else if (a.kde[l] >= 0) { dd = (uint32_t)key_pos(a.kde[l]); r |= W_DEXT; }
    return r | (m1 << W_M1_SHIFT) | (m4 << W_M4_SHIFT) | (dd << W_D_SHIFT);
}

// One-pass record choices of a multi-predecessor row (the batch kernel's
// adaptive fill). The predecessors arrive in the backtrack's priority order
// (in_weight descending, in-list position ascending), so each choice is the
// FIRST predecessor whose term equals the cell's final value. Per cell and
// per kind of term the fill keeps the running maximum of the terms seen so
// far and, in a 4-bit field, the in-list position of the first predecessor
// that reached it (a strict > keeps the first on ties):
//   y bits 0..3   dopen: first p with M_p + o1 at the max of those terms
//          4..7   dext : first p with D_p + e1 at the max of those terms
//          8..11  m4   : first p with M_p[j-1] + s at the diagonal max
//         12..15  m1   : first matching p (base_p == q[j-1]) at the max of
//                        the matching diagonal terms; 15 when that p fails
//                        the in_weight >= ind/10 rule (a later p may not
//                        take its place, src/align.cpp:1592-1604)
// 15 = none. A choice stands iff its maximum equals the final value (D for
// dopen/dext, M == Mpre for m4/m1), which is exactly "the first p whose term
// equals the final value". Positions must fit 4 bits: rows with more than
// TRACK_MAX_D in-window predecessors take the kernel's second pass instead.
constexpr int TRACK_MAX_D = 15;
constexpr uint32_t Y_NONE = 15u, Y_INIT = 0xffffu;
enum { Y_O = 0, Y_E = 4, Y_4 = 8, Y_1 = 12 };

PB_HD uint32_t y_set(uint32_t y, int sh, uint32_t v) { return (y & ~(15u << sh)) | (v << sh); }

// Vertical terms of one predecessor at one cell (the caller applies the
// vertical mask).
// The fields sit at bit `sh` of y (0, or 16 for the second cell of a pair
// that shares one register).
PB_HD void track_d(const Scoring& s, int32_t mb, int32_t db, uint32_t pos, int32_t& mO, int32_t& mE, uint32_t& y,
                   int sh = 0) {
    const int32_t co = add32(mb, s.o1), ce = add32(db, s.e1);
    if (co > mO) { mO = co; y = y_set(y, sh + Y_O, pos); }
    if (ce > mE) { mE = ce; y = y_set(y, sh + Y_E, pos); }
}

// Diagonal term `cand` of one predecessor at one cell (the caller applies the
// diagonal mask); pos4 / pos1 are the values recorded for m4 / m1 (Y_NONE
// where the backtrack never tests this term).
PB_HD void track_m(int32_t cand, bool bm, uint32_t pos4, uint32_t pos1, int32_t& mM, int32_t& m1, uint32_t& y,
                   int sh = 0) {
    if (cand > mM) { mM = cand; y = y_set(y, sh + Y_4, pos4); }
    if (bm && cand > m1) { m1 = cand; y = y_set(y, sh + Y_1, pos1); }
}

// The 4-byte record of one cell from the one-pass choices: own = own_flags,
// hm = (final M == Mpre), Mpre / Dv = the cell's diagonal / vertical maxima
// (clamped at NEG_INF as the fill initialises them).
PB_HD uint32_t track_record(uint32_t own, bool hm, int32_t Mpre, int32_t Dv, int32_t mM, int32_t m1, int32_t mO,
                            int32_t mE, uint32_t y) {
    const uint32_t n4 = (y >> Y_4) & 15u, n1 = (y >> Y_1) & 15u, nO = (y >> Y_O) & 15u, nE = (y >> Y_E) & 15u;
    const uint32_t m4v = (hm && mM == Mpre && n4 != Y_NONE) ? n4 : W_NONE;
    const uint32_t m1v = (hm && m1 == Mpre && n1 != Y_NONE) ? n1 : W_NONE;
    const bool okO = mO == Dv, okE = mE == Dv;
    uint32_t r = own & 15u;
    const uint32_t dd = okO ? nO : (okE ? nE : W_NONE);
    if (!okO && okE) r |= W_DEXT;
    return r | (m1v << W_M1_SHIFT) | (m4v << W_M4_SHIFT) | (dd << W_D_SHIFT);
}

// Decoded view of one record for the backtrack.
struct Rec {
    bool eqMD, eqMI, iopen, iext;
    int m1, m4, dpos;  // predecessor positions, -1 = none
    bool dext;
};
PB_HD Rec decode_small(uint8_t b) {
    Rec r;
    r.eqMD = b & R_EQMD; r.eqMI = b & R_EQMI; r.iopen = b & R_IOPEN; r.iext = b & R_IEXT;
    r.m1 = (b & R_M1) ? 0 : -1;
    r.m4 = (b & R_M4) ? 0 : -1;
    r.dpos = (b & (R_DOPEN | R_DEXT)) ? 0 : -1;
    r.dext = (b & R_DEXT) != 0;
    return r;
}
PB_HD Rec decode_wide(uint32_t w) {
    Rec r;
    r.eqMD = w & R_EQMD; r.eqMI = w & R_EQMI; r.iopen = w & R_IOPEN; r.iext = w & R_IEXT;
    uint32_t m1 = (w >> W_M1_SHIFT) & 511u, m4 = (w >> W_M4_SHIFT) & 511u, dd = (w >> W_D_SHIFT) & 511u;
    r.m1 = m1 == W_NONE ? -1 : (int)m1;
    r.m4 = m4 == W_NONE ? -1 : (int)m4;
    r.dpos = dd == W_NONE ? -1 : (int)dd;
    r.dext = (w & W_DEXT) != 0;
    return r;
}

// Backtrack move encoding: bits 0..2 query code, bits 3..4 kind, bits 5.. the
// predecessor row (window-local) for diagonal moves.
enum { MV_MATCH = 0, MV_MISMATCH = 1, MV_INSERT = 2 };
PB_HD int32_t mv_pack(int kind, int prow, int qc) { return (int32_t)(((uint32_t)prow << 5) | ((uint32_t)kind << 3) | (uint32_t)qc); }
PB_HD int mv_kind(int32_t v) { return (v >> 3) & 3; }
PB_HD int mv_row(int32_t v) { return (int)((uint32_t)v >> 5); }
PB_HD int mv_qc(int32_t v) { return v & 7; }

}  // namespace pb
