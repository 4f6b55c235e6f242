// ref_harness.cpp - drives the UNMODIFIED reference library (oracle/_ref/
// libminipoa.a, compiled from the reference's own sources) through the same
// loop as its main (src/main.cpp:84-126) and records every alignment() call.
// TEST INFRASTRUCTURE: it generates golden per-call records for the CPU
// restatement and for the CUDA path; it is never part of the product.
//
// Options are a subset of src/main.cpp:16-33: -M -X -O -E -b -f -B -S -k -w
// -W -t -r {0,1}; -d FILE writes per-read records:
//   A <read index> <score of the last poa() call> <path length>
//   <from>,<base>,<aligned_id> ...
// The score is the one poa() prints under verbose (src/align.cpp:1577); the
// harness captures std::cerr to read it.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "minipoa.h"

int main(int argc, char **argv) {
    para_t *para = new para_t();
    para->match = 2; para->mismatch = -4; para->gap_open1 = -4; para->gap_ext1 = -2;
    para->b = 100; para->f = 40; para->ab_band = false; para->k = 19; para->mm_w = 10;
    para->bw = 1000; para->progressive_poa = false; para->enable_seeding = false;
    para->thread = 1; para->result = 0; para->verbose = 0; para->poa_w = 0;  // -W read only when given (src/main.cpp:49-51)
    std::string in, dump;
    for (int a = 1; a < argc; a++) {
        std::string o = argv[a];
        auto nxt = [&]() { return std::atoi(argv[++a]); };
        if (o == "-B") para->ab_band = true;
        else if (o == "-S") para->enable_seeding = true;
        else if (o == "-M") para->match = nxt();
        else if (o == "-X") para->mismatch = nxt();
        else if (o == "-O") para->gap_open1 = nxt();
        else if (o == "-E") para->gap_ext1 = nxt();
        else if (o == "-b") para->b = nxt();
        else if (o == "-f") para->f = nxt();
        else if (o == "-k") para->k = nxt();
        else if (o == "-w") para->mm_w = nxt();
        else if (o == "-W") para->poa_w = nxt();
        else if (o == "-t") para->thread = nxt();
        else if (o == "-r") para->result = nxt();
        else if (o == "-d") dump = argv[++a];
        else in = o;
    }
    initPara(para);
    std::vector<seq_t> seqs;
    graph *DAG = new graph();
    DAG->init(para);
    readFile(seqs, in.c_str());
    minimizer_t *mm = new minimizer_t(para, seqs);
    aligned_buff_t *mpool = new aligned_buff_t[para->thread];
    FILE *df = dump.empty() ? nullptr : std::fopen(dump.c_str(), "w");
    for (size_t i = 0; i < seqs.size(); i++) {
        int rid = mm->ord[i];
        bool dp = DAG->node.size() > 2;
        std::stringstream cap;
        std::streambuf *old = std::cerr.rdbuf(cap.rdbuf());
        para->verbose = df ? 1 : 0;
        std::vector<res_t> res = alignment(para, DAG, mm, rid, seqs[rid].seq.c_str(), seqs[rid].seq.size(), mpool);
        para->verbose = 0;
        std::cerr.rdbuf(old);
        if (df && dp) {
            std::string line;
            long score = 0;
            while (std::getline(cap, line))
                if (line.compare(0, 6, "score:") == 0) score = std::atol(line.c_str() + 6);
            std::fprintf(df, "A %zu %ld %zu\n", i, score, res.size());
            for (size_t k = 0; k < res.size(); k++)
                std::fprintf(df, "%d,%d,%d%c", res[k].from, (int)res[k].base, res[k].aligned_id,
                             k + 1 == res.size() ? '\n' : ' ');
            if (res.empty()) std::fputc('\n', df);
        }
        DAG->add_path(para->m, (int)i, res, 1);
        DAG->topsort(para, i + 1 == seqs.size());
    }
    if (df) std::fclose(df);
    if (para->result == 0) DAG->output_consensus();
    else if (para->result == 1) DAG->output_rc_msa(para, mm->rid_to_ord, seqs);
    return 0;
}
