// ref_pool.cpp - runs the UNMODIFIED reference library (oracle/_ref/
// libminipoa.a, compiled from the reference's own sources) over many
// independent POA windows on a pool of host threads.
// TEST INFRASTRUCTURE: it makes the per-window consensus manifests that pin
// the batched CUDA engine at full benchmark size, and it is the CPU baseline
// the benchmark times. It is never part of the product.
//
// Each window is one minipoa run: the loop of src/main.cpp:84-121 (graph
// init, alignment() + add_path() + topsort() per read in input order), then
// graph::build_consensus (src/graph.cpp:294-350) and its `cons` string, which
// is what output_consensus prints (src/graph.cpp:352-357). Threads pull
// windows from an atomic counter (a continuously fed pool, no lock-step
// batches); each thread owns its aligned_buff_t arena, as src/main.cpp:109
// gives one per thread.
//
// Usage: ref_pool [-B] [-t threads] [-f first] [-n max_windows] [-s seconds] in.pwin out.cons
//   in.pwin   "PWIN" u32 n_windows, u32 n_reads, u32 win_off[n_windows+1],
//             u32 read_len[n_reads], then the reads' ASCII bases back to back
//   out.cons  per processed window in input order: u32 length, then the bases
//   -f / -n   process windows first .. first + max_windows - 1 only
//   -s        stop handing out windows after `seconds` (timing samples)
// Prints one line to stdout: "windows <n> seconds <wall> threads <t> prefix
// <p> busy <b>": windows done, the wall time of the pool (file I/O
// excluded), the length of the leading run of done windows written to
// out.cons, and the summed per-window thread time (windows * threads / busy
// is the pool's rate with every thread kept busy, free of the tail where
// the last windows finish on fewer threads).
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "minipoa.h"

static bool read_all(FILE* f, void* p, size_t n) { return std::fread(p, 1, n, f) == n; }

int main(int argc, char** argv) {
    bool ab = false;
    int threads = (int)std::thread::hardware_concurrency();
    long max_win = -1, first = 0;
    double seconds = -1.0;
    std::vector<std::string> pos;
    for (int a = 1; a < argc; a++) {
        std::string o = argv[a];
        if (o == "-B") ab = true;
        else if (o == "-t" && a + 1 < argc) threads = std::atoi(argv[++a]);
        else if (o == "-n" && a + 1 < argc) max_win = std::atol(argv[++a]);
        else if (o == "-f" && a + 1 < argc) first = std::atol(argv[++a]);
        else if (o == "-s" && a + 1 < argc) seconds = std::atof(argv[++a]);
        else pos.push_back(o);
    }
    if (pos.size() != 2 || threads < 1) {
        std::fprintf(stderr, "usage: ref_pool [-B] [-t threads] [-n max_windows] [-s seconds] in.pwin out.cons\n");
        return 2;
    }
    FILE* f = std::fopen(pos[0].c_str(), "rb");
    if (!f) { std::perror(pos[0].c_str()); return 2; }
    char magic[4];
    uint32_t nw = 0, nr = 0;
    if (!read_all(f, magic, 4) || std::memcmp(magic, "PWIN", 4) != 0 || !read_all(f, &nw, 4) || !read_all(f, &nr, 4)) {
        std::fprintf(stderr, "bad window file\n");
        return 2;
    }
    std::vector<uint32_t> win_off(nw + 1), rlen(nr);
    if (!read_all(f, win_off.data(), 4 * (size_t)(nw + 1)) || !read_all(f, rlen.data(), 4 * (size_t)nr)) {
        std::fprintf(stderr, "truncated window file\n");
        return 2;
    }
    std::vector<uint64_t> roff(nr + 1, 0);
    for (uint32_t r = 0; r < nr; r++) roff[r + 1] = roff[r] + rlen[r];
    std::string bases(roff[nr], '\0');
    if (!read_all(f, &bases[0], bases.size())) { std::fprintf(stderr, "truncated bases\n"); return 2; }
    std::fclose(f);
    if (first < 0 || (uint64_t)first > nw) { std::fprintf(stderr, "bad -f\n"); return 2; }
    const uint32_t avail = nw - (uint32_t)first;
    const uint32_t todo = max_win >= 0 && (uint64_t)max_win < avail ? (uint32_t)max_win : avail;

    // the CLI defaults of src/main.cpp:16-33 (-M 2 -X -4 -O -4 -E -2 -b 100 -f 40)
    para_t* para = new para_t();
    para->match = 2; para->mismatch = -4; para->gap_open1 = -4; para->gap_ext1 = -2;
    para->b = 100; para->f = 40; para->ab_band = ab; para->k = 19; para->mm_w = 10;
    para->bw = 1000; para->progressive_poa = false; para->enable_seeding = false;
    para->thread = 1; para->result = 0; para->verbose = 0; para->poa_w = 0;
    initPara(para);

    std::vector<std::string> cons(todo);
    std::vector<char> done(todo, 0);
    std::atomic<uint32_t> next(0);
    std::vector<double> busy(threads, 0.0);
    const auto t0 = std::chrono::steady_clock::now();
    auto elapsed = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    auto worker = [&](int tid) {
        aligned_buff_t mpool;
        while (true) {
            if (seconds >= 0.0 && elapsed() >= seconds) break;
            const uint32_t k = next.fetch_add(1);
            if (k >= todo) break;
            const double tw0 = elapsed();
            const uint32_t w = k + (uint32_t)first;
            std::vector<seq_t> seqs(win_off[w + 1] - win_off[w]);
            for (uint32_t r = win_off[w]; r < win_off[w + 1]; r++) {
                seq_t& s = seqs[r - win_off[w]];
                s.name = "seq" + std::to_string(r - win_off[w] + 1);
                s.seq.assign(bases, roff[r], rlen[r]);
            }
            graph* DAG = new graph();
            DAG->init(para);
            minimizer_t* mm = new minimizer_t(para, seqs);
            for (size_t i = 0; i < seqs.size(); i++) {
                const int rid = mm->ord[i];
                std::vector<res_t> res = alignment(para, DAG, mm, rid, seqs[rid].seq.c_str(),
                                                   (int)seqs[rid].seq.size(), &mpool);
                DAG->add_path(para->m, (int)i, res, 1);
                DAG->topsort(para, i + 1 == seqs.size());
            }
            DAG->build_consensus();
            cons[k] = DAG->cons;
            done[k] = 1;
            busy[tid] += elapsed() - tw0;
            delete mm;
            delete DAG;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) pool.emplace_back(worker, t);
    for (auto& t : pool) t.join();
    const double wall = elapsed();

    uint32_t ndone = 0;
    while (ndone < todo && done[ndone]) ndone++;
    FILE* o = std::fopen(pos[1].c_str(), "wb");
    if (!o) { std::perror(pos[1].c_str()); return 2; }
    for (uint32_t w = 0; w < ndone; w++) {
        const uint32_t n = (uint32_t)cons[w].size();
        std::fwrite(&n, 4, 1, o);
        std::fwrite(cons[w].data(), 1, n, o);
    }
    std::fclose(o);
    uint32_t total = 0;
    for (uint32_t w = 0; w < todo; w++) total += done[w];
    double busy_total = 0.0;
    for (double b : busy) busy_total += b;
    std::printf("windows %u seconds %.6f threads %d prefix %u busy %.6f\n", total, wall, threads, ndone, busy_total);
    return 0;
}
