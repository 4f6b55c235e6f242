// multi.cpp - one set of independent windows over several GPUs.
//
// Windows are independent (each is one minipoa run, src/main.cpp:84-126), so
// a window set shards with no exchange between devices: the windows are
// split by estimated cost, every device runs its share through its own
// context on its own host thread, and the consensus strings are gathered on
// the host in input order. No device reads another device's memory.
//
// Cost model: the DP of read k aligns ~k * len bases of graph against len
// query bases, so a window's work grows like bases * (reads + 1) - the same
// key the batch engine orders its windows by. The split is the longest-
// processing-time rule: windows by cost descending (input order on ties),
// each to the part with the least cost so far (lowest index on ties).
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/poa_b200.h"

namespace {

int64_t window_cost(const int32_t* read_len, const int32_t* win_off, int32_t w) {
    int64_t bases = 0;
    for (int32_t r = win_off[w]; r < win_off[w + 1]; r++) bases += read_len[r];
    return bases * (int64_t)(win_off[w + 1] - win_off[w] + 1);
}

int partition(const int32_t* read_len, const int32_t* win_off, int32_t n_windows, int32_t n_parts, int32_t* part,
              int64_t* part_cost);

}  // namespace

extern "C" int poa_batch_partition(const int32_t* read_len, const int32_t* win_off, int32_t n_windows,
                                   int32_t n_parts, int32_t* part, int64_t* part_cost) {
    if (!read_len || !win_off || !part || n_windows < 0 || n_parts < 1 || win_off[0] < 0) return POA_BAD_ARG;
    try {
        return partition(read_len, win_off, n_windows, n_parts, part, part_cost);
    } catch (const std::exception&) {
        return POA_OOM;
    }
}

namespace {

int partition(const int32_t* read_len, const int32_t* win_off, int32_t n_windows, int32_t n_parts, int32_t* part,
              int64_t* part_cost) {
    std::vector<int64_t> cost(n_windows);
    for (int32_t w = 0; w < n_windows; w++) {
        if (win_off[w + 1] < win_off[w]) return POA_BAD_ARG;
        cost[w] = window_cost(read_len, win_off, w);
    }
    std::vector<int32_t> order(n_windows);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return cost[a] > cost[b]; });
    std::vector<int64_t> load(n_parts, 0);
    for (int32_t w : order) {
        int32_t best = 0;
        for (int32_t g = 1; g < n_parts; g++)
            if (load[g] < load[best]) best = g;
        part[w] = best;
        load[best] += cost[w];
    }
    if (part_cost)
        for (int32_t g = 0; g < n_parts; g++) part_cost[g] = load[g];
    return POA_OK;
}

}  // namespace

namespace {

int consensus_multi(poa_ctx** ctxs, int32_t n_ctx, const uint8_t* seq, int64_t seq_bytes, const int64_t* read_off,
                    const int32_t* read_len, const int32_t* win_off, int32_t n_windows, char* cons,
                    int64_t cons_cap, int64_t* cons_off, int32_t* status);

}  // namespace

extern "C" int poa_batch_consensus_multi(poa_ctx** ctxs, int32_t n_ctx, const uint8_t* seq, int64_t seq_bytes,
                                         const int64_t* read_off, const int32_t* read_len, int32_t n_reads,
                                         const int32_t* win_off, int32_t n_windows, char* cons, int64_t cons_cap,
                                         int64_t* cons_off, int32_t* status) {
    if (!ctxs || n_ctx < 1 || !read_off || !read_len || !win_off || !cons_off || !status || n_windows < 0 ||
        n_reads < 0 || win_off[0] < 0 || win_off[n_windows] > n_reads || (cons_cap > 0 && !cons))
        return POA_BAD_ARG;
    try {
        return consensus_multi(ctxs, n_ctx, seq, seq_bytes, read_off, read_len, win_off, n_windows, cons, cons_cap,
                               cons_off, status);
    } catch (const std::exception&) {
        return POA_OOM;  // host memory or threads for the split ran out
    }
}

namespace {

int consensus_multi(poa_ctx** ctxs, int32_t n_ctx, const uint8_t* seq, int64_t seq_bytes, const int64_t* read_off,
                    const int32_t* read_len, const int32_t* win_off, int32_t n_windows, char* cons,
                    int64_t cons_cap, int64_t* cons_off, int32_t* status) {
    for (int32_t g = 0; g < n_ctx; g++)
        if (!ctxs[g]) return POA_BAD_ARG;
    std::vector<int32_t> part(n_windows);
    int st = poa_batch_partition(read_len, win_off, n_windows, n_ctx, part.data(), nullptr);
    if (st != POA_OK) return st;
    // each part's window list (input order) as its own read / window arrays over the shared bases
    struct Part {
        std::vector<int32_t> wins, win_off{0}, read_len, status;
        std::vector<int64_t> read_off, cons_off;
        std::vector<char> cons;
        int rc = POA_OK;
    };
    std::vector<Part> parts(n_ctx);
    for (int32_t w = 0; w < n_windows; w++) {
        Part& p = parts[part[w]];
        p.wins.push_back(w);
        for (int32_t r = win_off[w]; r < win_off[w + 1]; r++) {
            p.read_off.push_back(read_off[r]);
            p.read_len.push_back(read_len[r]);
        }
        p.win_off.push_back((int32_t)p.read_len.size());
    }
    std::vector<std::thread> threads;
    for (int32_t g = 0; g < n_ctx; g++) {
        Part& p = parts[g];
        if (p.wins.empty()) continue;
        p.rc = POA_OOM;  // until its thread has run
        auto job = [&p, g, ctxs, seq, seq_bytes, cons_cap]() {
            try {
                p.cons.resize((size_t)std::max<int64_t>(cons_cap, 1));
                p.cons_off.resize(p.wins.size() + 1);
                p.status.resize(p.wins.size());
            } catch (const std::exception&) {
                p.rc = POA_OOM;
                return;
            }
            p.rc = poa_batch_consensus(ctxs[g], seq, seq_bytes, p.read_off.data(), p.read_len.data(),
                                       (int32_t)p.read_len.size(), p.win_off.data(), (int32_t)p.wins.size(),
                                       p.cons.data(), (int64_t)p.cons.size(), p.cons_off.data(), p.status.data());
        };
        try {
            threads.emplace_back(job);
        } catch (const std::exception&) {
            job();  // no thread left: this part runs on the calling thread
        }
    }
    for (auto& t : threads) t.join();
    for (const Part& p : parts)
        if (p.rc != POA_OK) return p.rc;
    // gather in input order
    std::vector<int32_t> slot(n_windows);
    for (const Part& p : parts)
        for (size_t k = 0; k < p.wins.size(); k++) slot[p.wins[k]] = (int32_t)k;
    int64_t pos = 0;
    for (int32_t w = 0; w < n_windows; w++) {
        const Part& p = parts[part[w]];
        const int32_t k = slot[w];
        const int64_t len = p.cons_off[k + 1] - p.cons_off[k];
        cons_off[w] = pos;
        if (pos + len > cons_cap) return POA_BAD_ARG;
        if (len > 0) std::memcpy(cons + pos, p.cons.data() + p.cons_off[k], (size_t)len);
        pos += len;
        status[w] = p.status[k];
    }
    cons_off[n_windows] = pos;
    return POA_OK;
}

}  // namespace
