// driver.h - minipoa's per-read driver (src/main.cpp:84-126) and its
// alignment() dispatch (src/align.cpp:1741-1828) on top of a DP engine.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "graph.h"

namespace pb {

// para_t (include/parameter.h:5-19), the fields the path reads.
struct Params {
    int32_t match = 2, mismatch = -4, gap_open1 = -4, gap_ext1 = -2;  // src/main.cpp:18-21
    int32_t b = 100, f = 40;      // band, src/main.cpp:23-24
    int32_t ab_band = 0;          // -B
    int32_t enable_seeding = 0;   // -S
    int32_t k = 19, mm_w = 10;    // minimizer k-mer / window, src/main.cpp:27-28
    int32_t poa_w = 0;            // -W: read only when given (src/main.cpp:49-51), so 0 by default
    int32_t bw = 1000;            // src/main.cpp:65
    int32_t thread = 1;           // -t
    int32_t result = 0;           // -r: 0 consensus, 1 row-column MSA
    int32_t progressive = 0;      // -p
    int32_t verbose = 0;
};

// initPara sign rules, src/handle_input.cpp:45-51.
void normalize_params(Params& p);

Scoring scoring_of(const Params& p);

// One DP call: align q (codes 0..4) to the window; moves in backtrack order.
struct AlignOut {
    int32_t status = 0, score = 0;
    std::vector<int32_t> moves;
    int64_t cells = 0;
};

class DpEngine {
  public:
    virtual ~DpEngine() {}
    // Align several independent (window, query) pairs; every pair is one poa()
    // call. Implementations may run them concurrently.
    virtual void align_many(const std::vector<const HostWindow*>& wins,
                            const std::vector<const uint8_t*>& qs, const std::vector<int32_t>& qlens,
                            const std::vector<int32_t>& ab_bands, const Params& p,
                            std::vector<AlignOut>& outs) = 0;
};

// Host-side seeding for -S (minimizer anchors between the read and the current
// consensus, chained), src/minimizer.cpp:493-570 + src/lchain.cpp.
class Seeder;

// alignment(): returns a status; res gets the forward path.
int32_t alignment(const Params& p, Graph& g, Seeder* seeder, int rid, const uint8_t* q, int qlen,
                  DpEngine& eng, std::vector<Res>& res, std::vector<int32_t>* scores);

// The whole driver over reads (default order = input order unless -p).
// Returns status; text gets exactly what minipoa prints on stdout.
struct RunStats {
    int64_t cells = 0;
    int64_t dp_calls = 0;
};
// gfa (optional): the text of an existing graph to extend (-i, read_gfa,
// src/handle_input.cpp:444-494). Its paths come first in the outputs (as
// reads without bases), then the reads of seqs.
int32_t run_reads(const Params& p, const std::vector<std::string>& seqs,
                  const std::vector<std::string>& headers, DpEngine& eng, std::string& text,
                  std::vector<int32_t>* scores, RunStats* stats, const std::string* gfa = nullptr);

// read_gfa, src/handle_input.cpp:444-494: S lines add one node per base of the
// segment, P lines add their walk as a read (edges with the read's ord, in
// walk order; '-' walks linked from the sink side as the reference does); L
// and W lines are ignored; then an op-0 topsort. On error returns ST_BAD_ARG
// with the reason in err.
int32_t load_gfa(const Params& p, const std::string& text, Graph& g, std::vector<std::string>& path_names,
                 std::string& err);

}  // namespace pb
