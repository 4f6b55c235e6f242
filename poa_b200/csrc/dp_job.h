// dp_job.h - the unit of work of the DP kernels: one banded alignment of a
// query to a window of ranks [beg, end] of a POA graph (one poa() call,
// src/align.cpp:1353). Shared by the CUDA kernels, the host engine and the
// CPU model used by the tests.
#pragma once
#include <stdint.h>

#include "dp_core.h"

namespace pb {

// Rows are the window's ranks, row r = rank beg_i + r. All arrays are in the
// memory space of whoever runs the DP (device for the kernels).
struct WinView {
    int32_t n;                // rows (end_i - beg_i + 1)
    const int32_t* in_ptr;    // [n+1] CSR over in-window predecessors, in in-list order
    const int32_t* in_row;    // predecessor row
    const int32_t* in_w;      // in_weight of that edge
    const uint8_t* in_base;   // predecessor base as the DP sees it ('N' for row 0)
    const uint8_t* base;      // [n] node base of the row
    const int32_t* ind;       // [n] node in-degree count incl. repeats (include/node.h:26)
    const int32_t* hq;        // [n] hlen[rank] - hlen[beg_i]
    const int32_t* hq_loc;    // [n] hlen[r] - hlen[beg_i] (window-local index, src/align.cpp:1542)
    const int32_t* tq;        // [n] tlen[rank] - tlen[end_i]
    const int32_t* out_ptr;   // [n+1] CSR over in-window successors, in out-list order
    const int32_t* out_row;
};

// Adaptive-band state arrays (src/align.cpp:1375-1376), n entries each.
enum { AB_MP = 0, AB_SL, AB_PL, AB_PR, AB_OL, AB_OR, AB_OW, AB_NSTATE };

struct DpArgs {
    WinView v;
    const uint8_t* qs;   // qs[acj] = seq[acj-1] (qs[0] = 'N'), padded with 'N' (4)
    int32_t qlen;        // m = qlen + 1
    int32_t ab_band;     // adaptive band (only with f > 0)
    int32_t f, w;        // w = b + m/f (src/align.cpp:1378-1379)
    Scoring sc;
    RowMeta* meta;       // [n]
    int32_t* state;      // [AB_NSTATE * n] when adaptive
    int32_t* rs;         // row store: M/D blocks, 16 int32 per block
    int64_t rs_cap;      // int32 units
    // Row store layout. With ring_rows > 0 the first ring_rows * ring_blocks * 16
    // int32 are a ring of recent rows (row i in slot i % ring_rows). A row goes
    // to the spill area after the ring (bump-allocated) instead when one of its
    // in-window successors is ring_rows or more rows ahead, or when it is wider
    // than ring_blocks. ring_rows == 0 stores every row linearly. The static-band
    // plain kernel (plain_static.cuh) keeps its ring in shared memory instead
    // and stores only the other rows here, linearly.
    int32_t ring_rows, ring_blocks;
    uint8_t* tb;         // traceback records
    int64_t tb_cap;      // bytes
    int32_t* moves;      // backtrack moves (reverse order)
    int32_t moves_cap;
    int32_t* out;        // [0] status, [1] score, [2] number of moves, [3] cells
};

// Size of the shifted query buffer for a query of qlen bases.
PB_HD int64_t qs_bytes(int32_t qlen) {
    int64_t m = (int64_t)qlen + 1;
    int64_t need = (m / BLK + 3) * BLK;
    return (need + 15) / 16 * 16;
}

// Fill the shifted query buffer from encoded bases (0..4).
inline void make_qs(const uint8_t* q, int32_t qlen, uint8_t* qs) {
    int64_t len = qs_bytes(qlen);
    for (int64_t x = 0; x < len; x++) qs[x] = 4;
    for (int32_t k = 0; k < qlen; k++) qs[k + 2] = q[k];
}

}  // namespace pb
