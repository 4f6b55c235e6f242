// main.cpp - minipoa_b200, a drop-in for minipoa's command line
// (src/main.cpp:9-138): same options and defaults, same stdout, the DP on the
// GPU through the C ABI (include/poa_b200.h).
//
//   minipoa_b200 in.fa[.gz] [-M 2] [-X -4] [-O -4] [-E -2] [-b 100] [-f 40] [-B]
//                [-S] [-p] [-k 19] [-w 10] [-W 10000] [-t 1] [-r 0|1|2] [-i graph.gfa] [-V 0]
//
// Reads FASTA/FASTQ, optionally gzip-compressed (src/handle_input.cpp:13-43).
// -r 0 prints the consensus, -r 1 the row-column MSA, -r 2 the graph as GFA;
// -i extends the graph of a GFA file (its paths count as reads). Exit codes follow the
// reference: a backtrack that leaves the band exits 0 with no output
// (src/align.cpp:1584-1588), a backtrack error exits 1 (src/align.cpp:1730).
#include <zlib.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/poa_b200.h"
#include "reader.h"

namespace {

void usage() {
    std::cout << "minipoa_b200 <in.fa> [options]\n"
                 "  -M, --match INT        match score [2]\n"
                 "  -X, --mismatch INT     mismatch score [-4]\n"
                 "  -O, --gap_open INT     gap open [-4]\n"
                 "  -E, --gap_ext INT      gap extension [-2]\n"
                 "  -b, --band_b INT       band b [100]\n"
                 "  -f, --band_f INT       band f [40]\n"
                 "  -B, --ab_band          adaptive band\n"
                 "  -S, --seeding          minimizer seeding and anchoring\n"
                 "  -p, --progressive_poa  progressive read order (guide tree)\n"
                 "  -i, --inc_fp FILE      extend the graph of a GFA file\n"
                 "  -k, --k_mer INT        k-mer length [19]\n"
                 "  -w, --mm_w INT         minimizer window [10]\n"
                 "  -W, --poa_w INT        minimum distance between anchors [unset]\n"
                 "  -t, --thread INT       threads [1]\n"
                 "  -r, --result INT       0 consensus, 1 row-column MSA, 2 GFA [0]\n"
                 "  -V, --verbose INT      verbose level [0]\n"
                 "  -h, --help             this help\n";
}

}  // namespace

int main(int argc, char** argv) {
    poa_params p;
    poa_params_init(&p);
    std::string path, inc_fp;
    int32_t sample_num = 50;  // -s: parsed and unused, as in the reference (src/main.cpp:69-70)
    struct Opt {
        char s;
        const char* l;
        int32_t* v;
    } opts[] = {{'M', "match", &p.match},   {'X', "mismatch", &p.mismatch}, {'O', "gap_open", &p.gap_open},
                {'E', "gap_ext", &p.gap_ext}, {'b', "band_b", &p.band_b},     {'f', "band_f", &p.band_f},
                {'k', "k_mer", &p.k},        {'w', "mm_w", &p.mm_w},         {'W', "poa_w", &p.poa_w},
                {'t', "thread", &p.thread},   {'r', "result", &p.result},     {'V', "verbose", &p.verbose},
                {'s', "sample_num", &sample_num}};
    struct Flag {
        char s;
        const char* l;
        int32_t* v;
    } flags[] = {{'B', "ab_band", &p.ab_band}, {'S', "seeding", &p.seeding}, {'p', "progressive_poa", &p.progressive}};
    for (int a = 1; a < argc; a++) {
        std::string o = argv[a];
        if (o == "-h" || o == "--help") { usage(); return 0; }
        if (o.size() < 2 || o[0] != '-') { path = o; continue; }
        if (o == "-i" || o == "--inc_fp") {
            if (a + 1 >= argc) { std::cerr << "error parsing options: missing value for " << o << "\n"; return 1; }
            inc_fp = argv[++a];
            continue;
        }
        if (o.compare(0, 9, "--inc_fp=") == 0) { inc_fp = o.substr(9); continue; }
        if (o.compare(0, 2, "-i") == 0 && o.size() > 2) { inc_fp = o.substr(2); continue; }
        bool done = false;
        for (const Flag& f : flags)
            if (o == std::string("-") + f.s || o == std::string("--") + f.l) { *f.v = 1; done = true; }
        if (done) continue;
        for (const Opt& q : opts) {
            std::string sv;
            const std::string sh = std::string("-") + q.s, lg = std::string("--") + q.l;
            if (o == sh || o == lg) {
                if (a + 1 >= argc) { std::cerr << "error parsing options: missing value for " << o << "\n"; return 1; }
                sv = argv[++a];
            } else if (o.compare(0, 2, sh) == 0 && o.size() > 2 && o[1] == q.s) {
                sv = o.substr(2);
            } else if (o.compare(0, lg.size() + 1, lg + "=") == 0) {
                sv = o.substr(lg.size() + 1);
            } else {
                continue;
            }
            char* end = nullptr;
            long v = std::strtol(sv.c_str(), &end, 10);
            if (!end || *end) { std::cerr << "error parsing options: bad value " << sv << "\n"; return 1; }
            *q.v = (int32_t)v;
            done = true;
            break;
        }
        if (!done) { std::cerr << "error parsing options: unknown option " << o << "\n"; return 1; }
    }
    std::string data;
    if (!path.empty() && !pb::read_file(path.c_str(), data)) {
        std::cerr << "error read file: Error opening file " << path << std::endl;
        return 1;
    }
    std::vector<pb::SeqRec> recs = pb::parse_fastx(data);
    poa_ctx* ctx = poa_create(0, &p);
    if (!ctx) { std::cerr << "no usable CUDA device\n"; return 1; }
    std::vector<const char*> seqs(recs.size()), hdrs(recs.size());
    std::vector<int32_t> lens(recs.size());
    std::vector<std::string> hs(recs.size());
    for (size_t i = 0; i < recs.size(); i++) {
        seqs[i] = recs[i].seq.c_str();
        lens[i] = (int32_t)recs[i].seq.size();
        hs[i] = recs[i].name.empty() ? std::string() : recs[i].name + " " + recs[i].comment;
        hdrs[i] = hs[i].c_str();
    }
    char* text = nullptr;
    size_t tl = 0;
    int st;
    if (!inc_fp.empty()) {
        // an unreadable graph file leaves the graph empty, as read_gfa does (src/handle_input.cpp:453-455)
        std::string gfa;
        if (!pb::read_file(inc_fp.c_str(), gfa)) gfa.clear();
        st = poa_run_gfa(ctx, gfa.data(), gfa.size(), (int32_t)recs.size(), seqs.data(), lens.data(), hdrs.data(),
                         &text, &tl, nullptr);
    } else {
        st = poa_run(ctx, (int32_t)recs.size(), seqs.data(), lens.data(), hdrs.data(), &text, &tl, nullptr);
    }
    if (st == POA_BAND_ESCAPE) { poa_destroy(ctx); return 0; }
    if (st == POA_BT_FAIL) { std::cerr << " backtrack error" << "\n"; poa_destroy(ctx); return 1; }
    if (st != POA_OK) {
        std::cerr << "minipoa_b200: " << poa_status_str(st) << ": " << poa_last_error(ctx) << "\n";
        poa_destroy(ctx);
        return 1;
    }
    fwrite(text, 1, tl, stdout);
    poa_free(text);
    poa_destroy(ctx);
    return 0;
}
