// track_check.cpp - TEST-ONLY check of the batch kernel's one-pass record
// choices (dp_core.h track_d / track_m / track_record) against the generic
// per-predecessor comparisons flags_pred + encode_wide, which follow the
// reference backtrack's tests (src/align.cpp:1592-1604, 1632-1658) and are
// pinned by the golden cases through the CPU model.
//
// Random blocks: up to TRACK_MAX_D predecessors with random bands around the
// block, small value ranges (many ties), random bases, weights and left
// neighbours. The one-pass form is used by the kernel only where the fill's
// block-granular masks agree with the backtrack's per-cell test (no
// predecessor whose band starts inside the block, and, for cell 0, none whose
// previous block is in range but whose diagonal is masked), so only those
// cells are compared; the kernel recomputes the others with a second pass.
// Returns the number of mismatching cells (0 = pass).
#include <stdint.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <vector>

#include "dp_core.h"

using namespace pb;

namespace {

struct Rng {
    uint64_t s;
    uint32_t next() {
        s ^= s << 13; s ^= s >> 7; s ^= s << 17;
        return (uint32_t)(s >> 11);
    }
    int range(int lo, int hi) { return lo + (int)(next() % (uint32_t)(hi - lo + 1)); }
};

struct Pred {
    int Bs, Be, base, w, pos;
    int32_t Mb[BLK], Db[BLK], mprev;
};

}  // namespace

extern "C" int track_check(uint64_t seed, int blocks, int* compared) {
    Rng rng{seed * 2654435761u + 12345};
    const Scoring sc{2, -4, -6, -2};
    int bad = 0, cmp = 0;
    for (int t = 0; t < blocks; t++) {
        const int d = rng.range(2, TRACK_MAX_D);
        const int B = rng.range(0, 6);
        // row-local block index (0 = the row's first block), at most B
        const int b = (B == 0 || rng.range(0, 1)) ? 0 : std::min(B, rng.range(1, 4));
        const int ind = rng.range(1, 40);
        const int32_t base_v = rng.range(0, 1) ? NEG_INF : 100;
        std::vector<Pred> ps(d);
        for (int k = 0; k < d; k++) {
            Pred& p = ps[k];
            p.pos = k;
            p.Bs = rng.range(0, 4) ? rng.range(0, B) : rng.range(0, B + 2);
            p.Be = std::max(p.Bs + 1, rng.range(0, 4) ? B + rng.range(2, 5) : rng.range(1, B + 3));
            p.base = rng.range(0, 4);
            p.w = rng.range(1, 12);
            for (int l = 0; l < BLK; l++) {
                p.Mb[l] = base_v + rng.range(-8, 8);
                p.Db[l] = base_v + rng.range(-10, 6);
            }
            p.mprev = base_v + rng.range(-8, 8);
        }
        // the backtrack's priority order: in_weight descending, position ascending
        std::stable_sort(ps.begin(), ps.end(), [](const Pred& x, const Pred& y) { return x.w > y.w; });
        uint8_t qc8[BLK];
        for (int l = 0; l < BLK; l++) qc8[l] = (uint8_t)rng.range(0, 4);
        // pass 1 (reference form) and the one-pass tracking side by side
        int32_t Mpre[BLK], Dv[BLK];
        int32_t mM[BLK], m1[BLK], mO[BLK], mE[BLK];
        uint32_t y[BLK];
        for (int l = 0; l < BLK; l++) {
            Mpre[l] = Dv[l] = NEG_INF;
            mM[l] = m1[l] = mO[l] = mE[l] = INT_MIN;
            y[l] = Y_INIT;
        }
        bool slow = false, slow0 = false;
        for (const Pred& p : ps) {
            const PredMask mk = pred_mask(B, p.Bs, p.Be);
            const int32_t mprev = mk.prev_in ? p.mprev : NEG_INF;
            pass1_pred(sc, mk, b == 0, p.base, p.Mb, p.Db, mprev, qc8, Mpre, Dv);
            slow |= mk.blk_in && !mk.diag;
            slow0 |= mk.prev_in && !(mk.blk_in && mk.diag && b != 0);
            if (!mk.blk_in) continue;
            const uint32_t pos = (uint32_t)p.pos;
            const uint32_t p1 = p.w >= ind / 10 ? pos : Y_NONE;
            for (int l = 0; l < BLK; l++) track_d(sc, p.Mb[l], p.Db[l], pos, mO[l], mE[l], y[l]);
            if (!mk.diag) continue;
            for (int l = 0; l < BLK; l++) {
                const bool tracked = l > 0 || b != 0;
                const int32_t src0 = l == 0 ? (b == 0 ? NEG_INF : mprev) : p.Mb[l - 1];
                const bool bm = p.base == qc8[l];
                const int32_t cand = add32(src0, bm ? sc.match : sc.mismatch);
                track_m(cand, bm, tracked ? pos : Y_NONE, tracked ? p1 : Y_NONE, mM[l], m1[l], y[l]);
            }
        }
        if (slow) continue;
        // final M and I: a random horizontal value per cell, sometimes above H0
        int32_t M[BLK], I[BLK], H0[BLK];
        for (int l = 0; l < BLK; l++) {
            H0[l] = mx(Mpre[l], Dv[l]);
            I[l] = rng.range(0, 2) ? H0[l] + rng.range(-3, 1) : NEG_INF;
            M[l] = mx(H0[l], I[l]);
        }
        const int32_t Mleft = base_v + rng.range(-8, 8), Ileft = base_v + rng.range(-8, 8);
        for (int l = 0; l < BLK; l++) {
            if (l == 0 && slow0) continue;
            const int32_t mp = mx(NEG_INF, mM[l]), dv = mx(mx(NEG_INF, mO[l]), mE[l]);
            if (mp != Mpre[l] || dv != Dv[l]) { bad++; continue; }
            const int j = b * BLK + l;
            const uint32_t own = own_flags(sc, j, M[l], Dv[l], I[l], l ? M[l - 1] : Mleft, l ? I[l - 1] : Ileft);
            FlagAcc acc;
            flag_acc_init(acc);
            for (const Pred& p : ps) {
                const PredMask mk = pred_mask(B, p.Bs, p.Be);
                const int32_t mprev = mk.prev_in ? p.mprev : NEG_INF;
                flags_pred(sc, mk, p.base, p.w, p.pos, p.Mb, p.Db, mprev, qc8, M, Dv, acc);
            }
            const uint32_t want = encode_wide(own, acc, l, ind);
            const uint32_t got = track_record(own, M[l] == Mpre[l], Mpre[l], Dv[l], mM[l], m1[l], mO[l], mE[l], y[l]);
            cmp++;
            if (got != want) {
                if (bad < 5)
                    std::fprintf(stderr, "block %d cell %d: want %08x got %08x\n", t, l, want, got);
                bad++;
            }
        }
    }
    if (compared) *compared = cmp;
    return bad;
}
