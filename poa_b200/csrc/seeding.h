// seeding.h - host-side minimizer seeding and chaining for -S, and the
// progressive read order for -p. Restates minipoa's src/minimizer.cpp and
// src/lchain.cpp (themselves adapted from minimap2 and abPOA).
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

namespace pb {

struct Params;

// mm128_t (include/mmpriv.h:8). Minimizers: x = hash<<8 | span,
// y = rid<<32 | lastPos<<1 | strand. Anchors: x = rev<<63 | tid<<32 | tpos,
// y = flags<<40 | q_span<<32 | qpos.
struct Anchor {
    uint64_t x, y;
};

class Seeder {
  public:
    // minimizer_t::init, src/minimizer.cpp:159-194
    void init(const Params& p, const std::vector<std::string>& seqs);
    // minimizer_t::get_guide_tree, src/minimizer.cpp:195-386
    void guide_tree(const Params& p);
    // minimizer_t::collect_anchors_bycons, src/minimizer.cpp:537-570
    void anchors_by_consensus(const Params& p, int qid, int qlen, const std::string& cons,
                              std::vector<Anchor>& out);

    std::vector<int32_t> ord, rid_to_ord;

  private:
    int collect_anchors(int tid, int qid, int qlen, std::vector<Anchor>& anchors) const;
    void dp_chaining(const Params& p, std::vector<Anchor>& anchors, int tlen, int qlen);

    int nseq_ = 0;
    std::vector<Anchor> mm_, sorted_;  // all minimizers, and per-sequence copies sorted by x
    std::vector<int64_t> mm_h_;         // per-sequence offsets (nseq + 2 entries)
    std::vector<int32_t> len_;
    int maxl_ = 0;
};

// mm_sketch, src/minimizer.cpp:60-135 (forward strand only, no HPC).
void mm_sketch(const char* str, int len, int w, int k, uint32_t rid, std::vector<Anchor>& out);
// radix sort on x (include/ksort.h radix sort, 8-bit digits, stable per pass)
void radix_sort_x(Anchor* beg, Anchor* end);

}  // namespace pb
