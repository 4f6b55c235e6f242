// seeding.cpp - host-side minimizer seeding and chaining for -S.
//
// The anchors decide where minipoa splits a read into independently aligned
// sub-windows, so they are restated step for step: the (w,k)-minimizer sketch
// (src/minimizer.cpp:60-135, minimap2's sketch: forward strand only, no
// homopolymer compression), klib's in-place MSD radix sort (include/ksort.h:
// 101-150; not stable, so its exact permutation order is kept), the anchor
// merge join (src/minimizer.cpp:404-442), the local chaining DP with its
// backtrack and compaction (src/lchain.cpp:9-246, minimap2's lchain) and the
// global chain of local chains with the minimum-spacing filter
// (src/lchain.cpp:269-386, from abPOA). Float arithmetic follows the same
// expressions in the same order (IEEE single, no contraction).
//
// Lineage and licences: the algorithms restated here come, through minipoa
// (MIT, Copyright (c) 2025 Haodong Liu), from minimap2 (MIT, Heng Li; the
// sketch, mg_chain_bk_end, comput_sc, mg_lchain_dp and mg_log2) and klib's
// ksort.h (MIT, Copyright (c) 2008, 2011 Attractive Chaos; the radix sort),
// and from abPOA (MIT, Yan Gao; the chain of local chains). Bit-exact anchors
// need their exact steps, tie orders and float evaluation order.
#include "seeding.h"

#include <algorithm>
#include <cassert>
#include <cstring>

#include "driver.h"
#include "sketch.h"

namespace pb {

namespace {

constexpr int32_t kInf = 1000000000;  // src/lchain.cpp:8

// Cheap log2 for x >= 2 (include/mmpriv.h:12-20): exponent bits plus a
// quadratic fit of the mantissa.
inline float fast_log2(float x) {
    uint32_t i;
    std::memcpy(&i, &x, 4);
    float log_2 = (float)(int)((i >> 23) & 255) - 128;
    i &= ~(255u << 23);
    i += 127u << 23;
    float f;
    std::memcpy(&f, &i, 4);
    log_2 += (-0.34484843f * f + 2.02466578f) * f - 0.67487759f;
    return log_2;
}

void insertion_sort_x(Anchor* beg, Anchor* end) {
    for (Anchor* i = beg + 1; i < end; ++i) {
        if (i->x < (i - 1)->x) {
            Anchor tmp = *i;
            Anchor* j = i;
            for (; j > beg && tmp.x < (j - 1)->x; --j) *j = *(j - 1);
            *j = tmp;
        }
    }
}

struct Bucket {
    Anchor *b, *e;
};

void msd_radix(Anchor* beg, Anchor* end, int n_bits, int s) {
    const int size = 1 << n_bits, m = size - 1;
    Bucket bk[256];
    Bucket* be = bk + size;
    for (Bucket* k = bk; k != be; ++k) k->b = k->e = beg;
    for (Anchor* i = beg; i != end; ++i) ++bk[i->x >> s & m].e;
    for (Bucket* k = bk + 1; k != be; ++k) k->e += (k - 1)->e - beg, k->b = (k - 1)->e;
    // cycle-leader permutation into the buckets (American flag sort)
    for (Bucket* k = bk; k != be;) {
        if (k->b != k->e) {
            Bucket* l = bk + (k->b->x >> s & m);
            if (l != k) {
                Anchor tmp = *k->b, swp;
                do {
                    swp = tmp;
                    tmp = *l->b;
                    *l->b++ = swp;
                    l = bk + (tmp.x >> s & m);
                } while (l != k);
                *k->b++ = tmp;
            } else {
                ++k->b;
            }
        } else {
            ++k;
        }
    }
    bk[0].b = beg;
    for (Bucket* k = bk + 1; k != be; ++k) k->b = (k - 1)->e;
    if (s) {
        s = s > n_bits ? s - n_bits : 0;
        for (Bucket* k = bk; k != be; ++k) {
            if (k->e - k->b > 64) msd_radix(k->b, k->e, n_bits, s);
            else if (k->e - k->b > 1) insertion_sort_x(k->b, k->e);
        }
    }
}

// Chaining score between anchors (src/lchain.cpp:27-60) with the values the
// caller always passes: not cDNA, one segment, no equality filtering.
int32_t chain_score(const Anchor& ai, const Anchor& aj, int32_t max_dist_x, float pen_gap, float pen_skip) {
    const int32_t dq = (int32_t)ai.y - (int32_t)aj.y;
    if (dq <= 0 || dq > max_dist_x) return -kInf;
    const int32_t dr = (int32_t)(ai.x - aj.x);
    const int32_t dd = dr > dq ? dr - dq : dq - dr;
    const int32_t dg = dr < dq ? dr : dq;
    const int32_t q_span = (int32_t)(aj.y >> 32 & 0xff);
    int32_t sc = q_span < dg ? q_span : dg;
    if (dd || dg > q_span) {
        const float lin_pen = pen_gap * (float)dd + pen_skip * (float)dg;
        const float log_pen = dd >= 1 ? fast_log2((float)(dd + 1)) : 0.0f;
        if (dr == 0) ++sc;
        else sc -= (int)(lin_pen < log_pen ? lin_pen : log_pen);
    }
    return sc;
}

// src/lchain.cpp:9-25
int64_t chain_bk_end(int32_t max_drop, const Anchor* z, const int32_t* f, const int64_t* p, int32_t* t, int64_t k) {
    int64_t i = (int64_t)z[k].y, end_i = -1, max_i = i;
    int32_t max_s = 0;
    if (i < 0 || t[i] != 0) return i;
    do {
        int32_t s;
        t[i] = 2;
        end_i = i = p[i];
        s = i < 0 ? (int32_t)z[k].x : (int32_t)z[k].x - f[i];
        if (s > max_s) max_s = s, max_i = i;
        else if (max_s - s > max_drop) break;
    } while (i >= 0 && t[i] == 0);
    for (i = (int64_t)z[k].y; i >= 0 && i != end_i; i = p[i]) t[i] = 0;
    return max_i;
}

// src/lchain.cpp:63-142: pick chain ends by score, walk them back, keep
// chains with enough anchors and score. u[].x = strand|end tpos|end qpos,
// u[].y = [start, end) into v.
void chain_backtrack(int64_t n, const int32_t* f, const Anchor* a, const int64_t* p, std::vector<int32_t>& v,
                     std::vector<int32_t>& t, int32_t min_cnt, int32_t min_sc, int32_t max_drop,
                     std::vector<Anchor>& u, int32_t& n_v_out) {
    u.clear();
    n_v_out = 0;
    std::fill(t.begin(), t.end(), 0);
    int64_t n_z = 0;
    for (int64_t i = n - 1; i >= 0; i--) {
        // p[i] == -1 reads the int32 before t[] in the reference (src/lchain.cpp:74): the high
        // half of kalloc's block-size header, which is 0
        const int32_t tp = p[i] >= 0 ? t[p[i]] : 0;
        if (tp == 0 && f[i] >= 0 && f[i] >= min_sc) {
            ++n_z;
            t[i] = 2;
        }
        if (p[i] >= 0) t[p[i]] = 1;
    }
    if (n_z == 0) return;
    std::vector<Anchor> z(n_z);
    for (int64_t i = 0, k = 0; i < n; ++i)
        if (t[i] == 2) z[k].x = (uint64_t)(int64_t)f[i], z[k++].y = (uint64_t)i;
    radix_sort_x(z.data(), z.data() + n_z);
    std::fill(t.begin(), t.end(), 0);
    int64_t n_v = 0;
    for (int64_t k = n_z - 1; k >= 0; --k) {
        if (t[z[k].y] != 0) continue;
        const int64_t n_v0 = n_v;
        const int64_t end_i = chain_bk_end(max_drop, z.data(), f, p, t.data(), k);
        int64_t i;
        for (i = (int64_t)z[k].y; i != end_i; i = p[i]) v[n_v++] = (int32_t)i, t[i] = 1;
        const int32_t sc = i < 0 ? (int32_t)z[k].x : (int32_t)z[k].x - f[i];
        if (sc >= min_sc && n_v > n_v0 && n_v - n_v0 >= min_cnt) {
            const uint64_t end_id = z[k].y;
            const uint64_t strand = a[end_id].x >> 63, tpos = (uint32_t)a[end_id].x, qpos = (uint32_t)a[end_id].y;
            u.push_back(Anchor{strand << 63 | tpos << 32 | qpos, (uint64_t)n_v0 << 32 | (uint64_t)n_v});
        } else {
            n_v = n_v0;
        }
    }
    n_v_out = (int32_t)n_v;
}

// mg_lchain_dp (src/lchain.cpp:161-246): local chaining DP over anchors
// sorted by target position; returns the anchors of the kept chains, each
// chain in increasing order, and the chains themselves.
void local_chains(int max_dist_x, int max_dist_y, int bw, int max_skip, int max_iter, int min_cnt, int min_sc,
                  float pen_gap, float pen_skip, std::vector<Anchor>& a, std::vector<Anchor>& u) {
    (void)max_dist_y;
    u.clear();
    const int64_t n = (int64_t)a.size();
    if (n == 0) return;
    int32_t max_drop = bw;
    if (max_dist_x < bw) max_dist_x = bw;
    std::vector<int64_t> p(n);
    std::vector<int32_t> f(n), v(n), t(n, 0);
    int64_t st = 0, max_ii = -1;
    for (int64_t i = 0; i < n; ++i) {
        int64_t max_j = -1;
        int32_t max_f = (int32_t)(a[i].y >> 32 & 0xff), n_skip = 0, n_iter = 0;
        while (st < i && (a[i].x >> 32 != a[st].x >> 32 || a[i].x > a[st].x + (uint64_t)(int64_t)max_dist_x)) ++st;
        if (i - st > 5000) st = i - 5000;
        for (int64_t j = i - 1; j >= st; --j) {
            int32_t sc = chain_score(a[i], a[j], max_dist_x, pen_gap, pen_skip);
            if (sc == -kInf) continue;
            sc += f[j];
            if (sc > max_f) {
                max_f = sc, max_j = j;
                if (n_skip > 0) --n_skip;
            } else {
                if (sc != max_f) {
                    if (++n_iter > max_iter) break;
                }
                if (t[j] == (int32_t)i) {
                    if (++n_skip > max_skip) break;
                }
            }
            if (p[j] >= 0) t[p[j]] = (int32_t)i;
        }
        f[i] = max_f, p[i] = max_j;
        if (max_ii < 0 || (a[i].x - a[max_ii].x <= (uint64_t)(int64_t)max_dist_x && f[max_ii] < f[i])) max_ii = i;
    }
    int32_t n_v = 0;
    chain_backtrack(n, f.data(), a.data(), p.data(), v, t, min_cnt, min_sc, max_drop, u, n_v);
    if (u.empty()) {
        a.clear();
        return;
    }
    // compact_a, src/lchain.cpp:143-160
    std::vector<Anchor> b;
    b.reserve(n_v);
    for (const Anchor& c : u) {
        const int32_t s0 = (int32_t)(c.y >> 32), e0 = (int32_t)c.y;
        for (int32_t j = e0 - 1; j >= s0; j--) b.push_back(a[v[j]]);
    }
    a.swap(b);
}

// src/lchain.cpp:250-261
int32_t local_chain_score(int end_tpos_j, int end_qpos_j, int l, int r, const Anchor* a, const int32_t* score) {
    const int end_anchor_i = r;
    while (l + 1 < r) {
        const int mid = (l + r) / 2;
        const int tpos_mid = (int)(uint32_t)a[mid].x, qpos_mid = (int)(uint32_t)a[mid].y;
        if (tpos_mid <= end_tpos_j || qpos_mid <= end_qpos_j) l = mid;
        else r = mid;
    }
    if (r == end_anchor_i) return -kInf;
    return score[end_anchor_i - 1] - score[r];
}

// chain_dp (src/lchain.cpp:269-386): best global chain of local chains, then
// its anchors kept at least min_w apart on both sequences.
void global_chain(std::vector<Anchor>& lch, std::vector<Anchor>& a, int min_w, int tlen, int qlen, int max_dist_x,
                  float pen_gap, float pen_skip) {
    const int nl = (int)lch.size();
    std::vector<int32_t> f(a.size()), cs(nl), pre(nl);
    int gmax = -kInf, gi = -1;
    for (int i = 0, st = 0; i < nl; i++) {
        const uint64_t xi = lch[i].x, yi = lch[i].y;
        const int strand = (int)(xi >> 63);
        const int s_i = (int)(yi >> 32), e_i = (int32_t)yi;
        const int start_tpos_i = (int32_t)a[s_i].x, start_qpos_i = (int32_t)a[s_i].y;
        f[s_i] = (int32_t)(a[s_i].y >> 32 & 0xff);
        for (int j = s_i + 1; j < e_i; j++) f[j] = f[j - 1] + chain_score(a[j], a[j - 1], max_dist_x, pen_gap, pen_skip);
        int max_j = -1, max_score = f[e_i - 1];
        while (st < i) {
            if ((int)(lch[st].x >> 63) != strand) ++st;
            else break;
        }
        for (int j = i - 1; j >= st; --j) {
            const uint64_t xj = lch[j].x, yj = lch[j].y;
            const int end_tpos_j = (int)((xj >> 32) & 0x7fffffff), end_qpos_j = (int32_t)xj;
            const int s_j = (int)(yj >> 32);
            const int start_tpos_j = (int32_t)a[s_j].x;
            if (start_tpos_i < start_tpos_j) continue;
            int score1;
            if (start_tpos_i > end_tpos_j && start_qpos_i > end_qpos_j) score1 = cs[j] + f[e_i - 1];
            else score1 = cs[j] + local_chain_score(end_tpos_j, end_qpos_j, s_i, e_i, a.data(), f.data());
            if (score1 > max_score) max_score = score1, max_j = j;
        }
        cs[i] = max_score;
        pre[i] = max_j;
        if (max_score > gmax) gmax = max_score, gi = i;
    }
    std::vector<Anchor> out;
    if (gi < 0) {
        a.swap(out);  // no chain: the reference keeps the anchors list empty (src/lchain.cpp:328-330)
        return;
    }
    int cur_i = gi, pre_i = pre[gi];
    uint64_t cur_y = lch[cur_i].y;
    int last_tpos = tlen, last_qpos = qlen;
    int i = (int)(uint32_t)cur_y - 1;
    int filter_num = 0;
    while (pre_i != -1) {
        const uint64_t pre_x = lch[pre_i].x, pre_y = lch[pre_i].y;
        const int pre_end_tpos = (int)((pre_x >> 32) & 0x7fffffff), pre_end_qpos = (int32_t)pre_x;
        while (i >= 0) {
            const int cur_tpos = (int)a[i].x, cur_qpos = (int32_t)a[i].y;
            if (cur_tpos > pre_end_tpos && cur_qpos > pre_end_qpos) {
                if (last_tpos - cur_tpos >= min_w && last_qpos - cur_qpos >= min_w) {
                    if (filter_num < min_w / 10) a[i].y |= 1ULL << 40;  // MM_SEED_BAND_MODE_MASK, include/mmpriv.h:4
                    filter_num = 0;
                    out.push_back(a[i]);
                    last_tpos = cur_tpos, last_qpos = cur_qpos;
                } else {
                    filter_num++;
                }
            } else {
                break;
            }
            i--;
            if (i == (int)(cur_y >> 32)) break;
        }
        cur_i = pre_i, pre_i = pre[pre_i], cur_y = pre_y;
        i = (int)(uint32_t)cur_y - 1;
    }
    while (i >= 0) {
        const int cur_tpos = (int)a[i].x, cur_qpos = (int32_t)a[i].y;
        if (last_tpos - cur_tpos >= min_w && last_qpos - cur_qpos >= min_w) {
            if (filter_num < min_w / 10) a[i].y |= 1ULL << 40;
            filter_num = 0;
            out.push_back(a[i]);
            last_tpos = cur_tpos, last_qpos = cur_qpos;
        } else {
            filter_num++;
        }
        if (i == (int)(cur_y >> 32)) break;
        i--;
    }
    std::reverse(out.begin(), out.end());
    a.swap(out);
}

}  // namespace

void radix_sort_x(Anchor* beg, Anchor* end) {
    if (end - beg <= 64) insertion_sort_x(beg, end);
    else msd_radix(beg, end, 8, 56);
}

// src/minimizer.cpp:60-135 with is_hpc = 0 and the strand fixed to forward
// (:94-96): a minimizer for every w consecutive k-mers, ties broken towards
// the closest k-mer, identical k-mers within a window all reported.
void mm_sketch(const char* str, int len, int w, int k, uint32_t rid, std::vector<Anchor>& p) {
    if (len <= 0 || w <= 0 || w >= 256 || k <= 0 || k > 28) return;
    const uint64_t shift1 = 2 * (uint64_t)(k - 1), mask = (1ULL << 2 * k) - 1;
    uint64_t kmer[2] = {0, 0};
    int l = 0, buf_pos = 0, min_pos = 0, kmer_span = 0;
    Anchor buf[256], mn = {UINT64_MAX, UINT64_MAX};
    for (int j = 0; j < w; j++) buf[j] = Anchor{UINT64_MAX, UINT64_MAX};
    for (int i = 0; i < len; ++i) {
        const int c = nt4((uint8_t)str[i]);
        Anchor info = {UINT64_MAX, UINT64_MAX};
        if (c < 4) {
            kmer_span = l + 1 < k ? l + 1 : k;
            kmer[0] = (kmer[0] << 2 | (uint64_t)c) & mask;
            kmer[1] = (kmer[1] >> 2) | (3ULL ^ (uint64_t)c) << shift1;
            ++l;
            if (l >= k && kmer_span < 256) {
                info.x = hash64(kmer[0], mask) << 8 | (uint64_t)kmer_span;
                info.y = (uint64_t)rid << 32 | (uint64_t)(uint32_t)i << 1;
            }
        } else {
            l = 0, kmer_span = 0;
        }
        buf[buf_pos] = info;
        if (l == w + k - 1 && mn.x != UINT64_MAX) {  // first full window: identical k-mers not stored yet
            for (int j = buf_pos + 1; j < w; ++j)
                if (mn.x == buf[j].x && buf[j].y != mn.y) p.push_back(buf[j]);
            for (int j = 0; j < buf_pos; ++j)
                if (mn.x == buf[j].x && buf[j].y != mn.y) p.push_back(buf[j]);
        }
        if (info.x <= mn.x) {  // a new minimum; the old one is written out
            if (l >= w + k && mn.x != UINT64_MAX) p.push_back(mn);
            mn = info, min_pos = buf_pos;
        } else if (buf_pos == min_pos) {  // the minimum left the window
            if (l >= w + k - 1 && mn.x != UINT64_MAX) p.push_back(mn);
            mn.x = UINT64_MAX;
            for (int j = buf_pos + 1; j < w; ++j)
                if (mn.x >= buf[j].x) mn = buf[j], min_pos = j;
            for (int j = 0; j <= buf_pos; ++j)
                if (mn.x >= buf[j].x) mn = buf[j], min_pos = j;
            if (l >= w + k - 1 && mn.x != UINT64_MAX) {
                for (int j = buf_pos + 1; j < w; ++j)
                    if (mn.x == buf[j].x && mn.y != buf[j].y) p.push_back(buf[j]);
                for (int j = 0; j <= buf_pos; ++j)
                    if (mn.x == buf[j].x && mn.y != buf[j].y) p.push_back(buf[j]);
            }
        }
        if (++buf_pos == w) buf_pos = 0;
    }
    if (mn.x != UINT64_MAX) p.push_back(mn);
}

// minimizer_t::init / collect_mm, src/minimizer.cpp:142-194
void Seeder::init(const Params& p, const std::vector<std::string>& seqs) {
    nseq_ = (int)seqs.size();
    ord.resize(nseq_);
    rid_to_ord.resize(nseq_);
    for (int i = 0; i < nseq_; i++) ord[i] = rid_to_ord[i] = i;
    mm_.clear();
    sorted_.clear();
    mm_h_.assign(nseq_ + 2, 0);
    len_.resize(nseq_);
    maxl_ = 0;
    if (!(p.progressive || p.enable_seeding)) return;
    for (int i = 0; i < nseq_; i++) {
        mm_sketch(seqs[i].data(), (int)seqs[i].size(), p.mm_w, p.k, (uint32_t)i, mm_);
        mm_h_[i + 1] = (int64_t)mm_.size();
        len_[i] = (int32_t)seqs[i].size();
        maxl_ = std::max(maxl_, len_[i]);
    }
    if (p.enable_seeding) {
        sorted_ = mm_;
        for (int i = 0; i < nseq_; i++) radix_sort_x(sorted_.data() + mm_h_[i], sorted_.data() + mm_h_[i + 1]);
    }
}

// minimizer_t::get_guide_tree, src/minimizer.cpp:195-386: the progressive read
// order of -p. Shared minimizers per read pair (for every hash, the smaller of
// the two reads' counts), a length-weighted Jaccard similarity per ordered
// pair, the most similar pair first, then repeatedly the read with the largest
// similarity sum to the reads already ordered (first maximum wins). Pairs are
// counted over the reads present in each hash group only, which adds the same
// totals as the reference's loop over all pairs.
void Seeder::guide_tree(const Params& p) {
    const int n = nseq_;
    if (!p.progressive || n < 2 || mm_.empty()) return;
    std::vector<Anchor> mm = mm_;
    std::sort(mm.begin(), mm.end(), [](const Anchor& a, const Anchor& b) { return a.x < b.x; });
    auto tri = [](int64_t hi, int64_t lo) { return ((hi * (hi + 1)) >> 1) + lo; };
    std::vector<int32_t> hit((size_t)tri(n - 1, n - 1) + 1, 0);
    std::vector<int32_t> cnt(n, 0), present;
    for (size_t a = 0; a < mm.size();) {
        size_t b = a;
        while (b < mm.size() && mm[b].x == mm[a].x) b++;
        present.clear();
        for (size_t j = a; j < b; j++) {
            const int r = (int)(mm[j].y >> 32);
            if (cnt[r]++ == 0) present.push_back(r);
            hit[tri(r, r)]++;
        }
        for (size_t u = 0; u < present.size(); u++)
            for (size_t v = u + 1; v < present.size(); v++) {
                const int r1 = std::min(present[u], present[v]), r2 = std::max(present[u], present[v]);
                hit[tri(r2, r1)] += std::min(cnt[r1], cnt[r2]);
            }
        for (int r : present) cnt[r] = 0;
        a = b;
    }
    std::vector<double> jac((size_t)n * n, 0.0);
    double max_jac = -1.0;
    int max_i = -1, max_j = -1;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            if (i == j) continue;
            const int shared = i > j ? hit[tri(i, j)] : hit[tri(j, i)];
            const int tot = hit[tri(i, i)] + hit[tri(j, j)] - shared;
            double v = 0.0;
            if (tot > 0) {
                v = (0.0 + shared) / tot;
                v = v * ((0.51 * len_[i] / maxl_) + (0.49 * len_[j] / maxl_));
            }
            jac[(size_t)i * n + j] = v;
            if (v > max_jac) { max_jac = v; max_i = i; max_j = j; }
        }
    std::vector<char> in_ord(n, 0);
    ord[0] = max_i;
    ord[1] = max_j;
    rid_to_ord[max_i] = 0;
    rid_to_ord[max_j] = 1;
    in_ord[max_i] = in_ord[max_j] = 1;
    for (int k = 2; k < n; k++) {
        double best = -1.0;
        int pick = n;
        for (int r2 = 0; r2 < n; r2++) {
            if (in_ord[r2]) continue;  // the reference scores it -1, which never wins
            double sum = 0.0;
            for (int t = 0; t < k; t++) sum += jac[(size_t)ord[t] * n + r2];
            if (sum > best) { best = sum; pick = r2; }
        }
        ord[k] = pick;
        rid_to_ord[pick] = k;
        in_ord[pick] = 1;
    }
}

// src/minimizer.cpp:404-442: same-hash minimizer pairs of target tid and
// query qid; anchors sorted by target position
int Seeder::collect_anchors(int tid, int qid, int qlen, std::vector<Anchor>& anchors) const {
    int64_t i = mm_h_[tid], j = mm_h_[qid];
    const int64_t ie = mm_h_[tid + 1], je = mm_h_[qid + 1];
    int64_t jj = j;
    while (i < ie && j < je) {
        const uint64_t xi = sorted_[i].x, xj = sorted_[j].x;
        if (xi == xj) {
            int64_t ii = i;
            for (; ii < ie; ++ii) {
                if (sorted_[ii].x != xi) break;
                const uint64_t yi = sorted_[ii].y;
                for (jj = j; jj < je; ++jj) {
                    const uint64_t xjj = sorted_[jj].x;
                    if (xjj != xj) break;
                    const uint64_t yj = sorted_[jj].y;
                    const uint32_t qspan = (uint32_t)(xjj & 0xff);
                    Anchor an;
                    if ((yi & 1) == (yj & 1)) {
                        an.x = (yi & 0x7fffffff00000000ULL) | ((uint32_t)yi >> 1);
                        an.y = (uint64_t)qspan << 32 | ((uint32_t)yj >> 1);
                    } else {
                        an.x = 1ULL << 63 | (yi & 0xffffffff00000000ULL) | ((uint32_t)yi >> 1);
                        an.y = (uint64_t)qspan << 32 | (uint32_t)(qlen - (int)(((uint32_t)yj >> 1) + 1 - qspan) - 1);
                    }
                    anchors.push_back(an);
                }
            }
            i = ii, j = jj;
        } else if (xi < xj) {
            ++i;
        } else {
            ++j;
        }
    }
    radix_sort_x(anchors.data(), anchors.data() + anchors.size());
    return (int)anchors.size();
}

// src/minimizer.cpp:493-535
void Seeder::dp_chaining(const Params& p, std::vector<Anchor>& anchors, int tlen, int qlen) {
    int min_w = std::min(20000, (tlen + 24 - 1) / 24);
    if (p.poa_w) min_w = std::min(min_w, p.poa_w + p.k);
    const int max_bw = p.bw, max_dis = max_bw;
    const float pen_gap = (float)(0.01 * p.k), pen_skip = (float)(0.0 * 0.01 * p.k);
    std::vector<Anchor> lch;
    local_chains(max_dis, max_dis, max_bw, 25, 50, 3, 100, pen_gap, pen_skip, anchors, lch);
    if (lch.empty()) {
        anchors.clear();
        return;
    }
    radix_sort_x(lch.data(), lch.data() + lch.size());
    global_chain(lch, anchors, min_w, tlen, qlen, max_dis, pen_gap, pen_skip);
}

// src/minimizer.cpp:537-570: sketch the current consensus as sequence nseq,
// anchor the query against it, chain.
void Seeder::anchors_by_consensus(const Params& p, int qid, int qlen, const std::string& cons,
                                  std::vector<Anchor>& out) {
    const int n = nseq_;
    mm_.resize(mm_h_[n]);
    mm_sketch(cons.data(), (int)cons.size(), p.mm_w, p.k, (uint32_t)n, mm_);
    mm_h_[n + 1] = (int64_t)mm_.size();
    sorted_.resize(mm_h_[n]);
    sorted_.insert(sorted_.end(), mm_.begin() + mm_h_[n], mm_.end());
    radix_sort_x(sorted_.data() + mm_h_[n], sorted_.data() + mm_h_[n + 1]);
    out.clear();
    collect_anchors(n, qid, qlen, out);
    dp_chaining(p, out, (int)cons.size(), qlen);
}

}  // namespace pb
