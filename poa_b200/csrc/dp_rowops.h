// dp_rowops.h - the serial per-row steps of the DP, executed by one thread on
// the device (and by the CPU model in the tests): band selection, the
// adaptive-band update after a row, and the record-driven backtrack.
#pragma once
#include "dp_job.h"

namespace pb {

// Band of row i, src/align.cpp:1382-1390 (static / full) and :1410-1414,
// :1433-1444 (adaptive, f > 0 && ab_band).
PB_HD void row_band(const DpArgs& a, int i, int m, int& Bs, int& Be) {
    if (a.f > 0 && a.ab_band) {
        const int n = a.v.n;
        const int32_t* st = a.state;
        band_adaptive(a.v.hq[i], a.v.tq[i], m, a.w, st[AB_PL * n + i], st[AB_PR * n + i],
                      st[AB_OL * n + i], st[AB_OR * n + i], st[AB_OW * n + i], Bs, Be);
    } else {
        band_static(a.f, a.v.hq[i], a.v.tq[i], m, a.w, Bs, Be);
    }
}

// Adaptive-band bookkeeping after row i (i >= 1), src/align.cpp:1516-1568.
// max_j is the first argmax of the row's final M over its computed cells.
PB_HD void adaptive_update(const DpArgs& a, int i, int Bs, int max_j) {
    const int n = a.v.n;
    int32_t* Mp = a.state + AB_MP * n;
    int32_t* Sl = a.state + AB_SL * n;
    int32_t* Pl = a.state + AB_PL * n;
    int32_t* Pr = a.state + AB_PR * n;
    int32_t* Ol = a.state + AB_OL * n;
    int32_t* Or = a.state + AB_OR * n;
    int32_t* Ow = a.state + AB_OW * n;
    int max_acj = Bs * BLK + max_j, max_slp = 0;
    bool is_match = false;
    Mp[i] = max_acj;
    if ((int)a.v.base[i] == (int)a.qs[max_acj + 1]) {  // cur.base == seq[max_acj]
        for (int e = a.v.in_ptr[i]; e < a.v.in_ptr[i + 1]; e++) {
            int p = a.v.in_row[e];
            max_slp = Sl[p] > max_slp ? Sl[p] : max_slp;
            if (Mp[p] + 1 == Mp[i]) {
                Sl[i] = mx(Sl[i], Sl[p] + 1);
                is_match = true;
            }
        }
    }
    if (!is_match && max_slp < 30) {
        Ow[i] += max_slp + 1;
        Ow[i] = mn(Ow[i], 5 * a.w);
    }
    const int o0 = a.v.out_ptr[i], o1 = a.v.out_ptr[i + 1];
    if (Sl[i] >= 30) {
        Ol[i] = max_acj - a.v.hq_loc[i];
        Or[i] = max_acj - a.v.hq_loc[i];
        Ow[i] = 0;
        for (int e = o0; e < o1; e++) {
            int s = a.v.out_row[e];
            Ol[s] = Ol[i];
            Or[s] = Or[i];
        }
    }
    for (int e = o0; e < o1; e++) {
        int s = a.v.out_row[e];
        Ol[s] = mn(Ol[s], Ol[i]);
        Or[s] = mx(Or[s], Or[i]);
    }
    for (int e = o0; e < o1; e++) {
        int s = a.v.out_row[e];
        Pl[s] = mn(Pl[s], max_acj);
        Pr[s] = mx(Pr[s], max_acj + 1);
        Ow[s] = Ow[i] ? mx(Ow[s], Ow[i]) : Ow[i];
    }
}

// Initialise the adaptive state, src/align.cpp:1375-1376 (Pl = m, rest 0).
PB_HD void adaptive_init_entry(const DpArgs& a, int r, int m) {
    const int n = a.v.n;
    for (int k = 0; k < AB_NSTATE; k++) a.state[k * n + r] = 0;
    a.state[AB_PL * n + r] = m;
}

// Backtrack from (n-1, m) over the records, src/align.cpp:1572-1736. Moves
// are written in backtrack order (the host reverses them). Returns a status.
PB_HD int32_t backtrack_records(const DpArgs& a, int m, int32_t& nmoves) {
    int i = a.v.n - 1, acj = m, op = ALL_OP;
    int32_t nm = 0;
    while (i > 0 || acj > 0) {
        const RowMeta rm = a.meta[i];
        if (acj > (rm.Be - 1) * BLK || acj < rm.Bs * BLK) { nmoves = nm; return ST_BAND_ESCAPE; }
        const int j = acj - rm.Bs * BLK;
        const int bn = rm.Be - rm.Bs - 1;
        if (j >= bn * BLK) { nmoves = nm; return ST_BT_FAIL; }  // the pad cell; no move lands there
        const int e0 = a.v.in_ptr[i];
        const int d = a.v.in_ptr[i + 1] - e0;
        const Rec r = d >= 2 ? decode_wide(*(const uint32_t*)(a.tb + rm.tb + (int64_t)j * 4))
                             : decode_small(a.tb[rm.tb + j]);
        if (nm + 1 > a.moves_cap) { nmoves = nm; return ST_OOM; }
        const int qc = acj > 0 ? a.qs[acj] : 4;
        if ((op & M_OP) && acj > 0 && r.m1 >= 0) {
            int p = a.v.in_row[e0 + r.m1];
            int kind = (int)a.v.in_base[e0 + r.m1] == qc ? MV_MATCH : MV_MISMATCH;
            a.moves[nm++] = mv_pack(kind, p, qc);
            op = ALL_OP; i = p; acj--;
            continue;
        }
        if ((op & D_OP) && (op == D_OP || r.eqMD) && r.dpos >= 0) {
            i = a.v.in_row[e0 + r.dpos];
            op = r.dext ? D_OP : (M_OP | I_OP);
            continue;
        }
        if ((op & I_OP) && acj > 0 && j >= 1 && (op == I_OP || r.eqMI)) {
            if (r.iopen) { a.moves[nm++] = mv_pack(MV_INSERT, 0, qc); op = M_OP | D_OP; acj--; continue; }
            if (r.iext) { a.moves[nm++] = mv_pack(MV_INSERT, 0, qc); op = I_OP; acj--; continue; }
        }
        if ((op & M_OP) && acj > 0 && r.m4 >= 0) {
            int p = a.v.in_row[e0 + r.m4];
            int kind = (int)a.v.in_base[e0 + r.m4] == qc ? MV_MATCH : MV_MISMATCH;
            a.moves[nm++] = mv_pack(kind, p, qc);
            op = ALL_OP; i = p; acj--;
            continue;
        }
        nmoves = nm;
        return ST_BT_FAIL;
    }
    nmoves = nm;
    return ST_OK;
}

}  // namespace pb
