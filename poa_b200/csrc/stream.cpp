// stream.cpp - windows read from files, parsed on host threads while the
// device runs the previous chunk.
//
// Each window is one file, exactly what one minipoa run reads: FASTA or
// FASTQ, optionally gzip-compressed (src/handle_input.cpp:13-43, kseq over
// gzread). The reads keep their order and bases as written (encoding happens
// on the device). Files are taken in chunks of `chunk` windows: host threads
// read and parse chunk k+1 into a page-locked staging buffer while chunk k
// is uploaded, run (with the proposer's plan when the context has one) and
// downloaded, so the parse of every chunk but the first is hidden behind
// device work. The chunk should hold several times the engine's resident
// windows (slots), or the persistent launch runs short of work at its end.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdint>
#include <cstring>
#include <future>
#include <string>
#include <thread>
#include <vector>

#include "../../include/poa_b200.h"
#include "reader.h"

namespace {

// One chunk of windows in the batch layout, its bases in page-locked memory.
struct Chunk {
    uint8_t* seq = nullptr;
    int64_t cap = 0, bytes = 0;
    std::vector<int64_t> read_off;
    std::vector<int32_t> read_len, win_off;
    int rc = POA_OK;
    ~Chunk() {
        if (seq) poa_free_pinned(seq);
    }
};

void parse_chunk_body(const char* const* paths, int32_t w0, int32_t w1, int threads, Chunk& c) {
    const int32_t nw = w1 - w0;
    std::vector<std::vector<pb::SeqRec>> recs(nw);
    std::vector<char> ok(nw, 1);
    std::atomic<int32_t> next(0);
    std::atomic<bool> oom(false);
    auto work = [&]() {
        try {
            std::string text;
            for (int32_t k = next++; k < nw; k = next++) {
                text.clear();
                if (!pb::read_file(paths[w0 + k], text)) { ok[k] = 0; continue; }
                recs[k] = pb::parse_fastx(text);
            }
        } catch (const std::exception&) {
            oom = true;
            next = nw;  // the other threads stop too
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; t++) {
        try {
            pool.emplace_back(work);
        } catch (const std::exception&) {
            break;  // fewer host threads; the calling thread still parses
        }
    }
    work();
    for (auto& t : pool) t.join();
    if (oom) { c.rc = POA_OOM; return; }
    c.read_off.clear();
    c.read_len.clear();
    c.win_off.assign(1, 0);
    int64_t bytes = 0;
    for (int32_t k = 0; k < nw; k++) {
        if (!ok[k]) { c.rc = POA_BAD_ARG; return; }
        for (const pb::SeqRec& r : recs[k]) {
            if (r.seq.size() > (size_t)INT32_MAX) { c.rc = POA_BAD_ARG; return; }
            bytes += (int64_t)r.seq.size();
        }
    }
    if (bytes + 16 > c.cap) {
        if (c.seq) poa_free_pinned(c.seq);
        c.cap = (bytes + 16) * 5 / 4;
        c.seq = (uint8_t*)poa_alloc_pinned((size_t)c.cap);
        if (!c.seq) { c.cap = 0; c.rc = POA_OOM; return; }
    }
    int64_t pos = 0;
    for (int32_t k = 0; k < nw; k++) {
        for (const pb::SeqRec& r : recs[k]) {
            if (!r.seq.empty()) std::memcpy(c.seq + pos, r.seq.data(), r.seq.size());
            c.read_off.push_back(pos);
            c.read_len.push_back((int32_t)r.seq.size());
            pos += (int64_t)r.seq.size();
        }
        c.win_off.push_back((int32_t)c.read_len.size());
    }
    c.bytes = pos;
    c.rc = POA_OK;
}

// A chunk that could not be built (host memory, an unreadable file) carries
// its status in rc; nothing escapes to the caller's thread as an exception.
void parse_chunk(const char* const* paths, int32_t w0, int32_t w1, int threads, Chunk& c) {
    c.rc = POA_OK;
    try {
        parse_chunk_body(paths, w0, w1, threads, c);
    } catch (const std::exception&) {
        c.rc = POA_OOM;
    }
}

}  // namespace

extern "C" int poa_batch_consensus_files(poa_ctx* ctx, const char* const* paths, int32_t n_files, int32_t chunk,
                                         int32_t threads, char* cons, int64_t cons_cap, int64_t* cons_off,
                                         int32_t* status) {
    if (!ctx || !paths || n_files < 0 || chunk < 1 || !cons_off || !status || (cons_cap > 0 && !cons))
        return POA_BAD_ARG;
    for (int32_t w = 0; w < n_files; w++)
        if (!paths[w]) return POA_BAD_ARG;
    if (threads < 1) threads = std::max(1, (int)std::thread::hardware_concurrency());
    Chunk bufs[2];
    cons_off[0] = 0;
    if (n_files == 0) return POA_OK;
    parse_chunk(paths, 0, std::min(chunk, n_files), threads, bufs[0]);
    int64_t pos = 0;
    int k = 0;
    for (int32_t w0 = 0; w0 < n_files; w0 += chunk, k ^= 1) {
        Chunk& cur = bufs[k];
        if (cur.rc != POA_OK) return cur.rc;
        const int32_t w1 = std::min(n_files, w0 + chunk);
        // the next chunk is read and parsed while this one is on the device
        std::future<void> next;
        if (w1 < n_files) {
            try {
                next = std::async(std::launch::async, parse_chunk, paths, w1, std::min(n_files, w1 + chunk),
                                  threads, std::ref(bufs[k ^ 1]));
            } catch (const std::exception&) {
                parse_chunk(paths, w1, std::min(n_files, w1 + chunk), threads, bufs[k ^ 1]);  // no thread: now
            }
        }
        const int32_t nw = w1 - w0;
        int rc = poa_batch_upload(ctx, cur.seq, cur.bytes, cur.read_off.data(), cur.read_len.data(),
                                  (int32_t)cur.read_len.size(), cur.win_off.data(), nw);
        if (rc == POA_OK) rc = poa_batch_run(ctx, nullptr);
        if (rc == POA_OK) rc = poa_batch_download(ctx, cons + pos, cons_cap - pos, cons_off + w0, status + w0);
        if (next.valid()) next.wait();
        if (rc != POA_OK) return rc;
        // the chunk's offsets are relative to its own start
        for (int32_t w = w0; w <= w1; w++) cons_off[w] += pos;
        pos = cons_off[w1];
    }
    return POA_OK;
}
