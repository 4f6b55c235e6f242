// gpu_engine.cu - host side of the plain DP path (see gpu_engine.h).
#include "gpu_engine.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <stdexcept>

#include "plain.cuh"
#include "plain_static.cuh"

namespace pb {

void cuda_check(int err, const char* what) {
    if (err != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString((cudaError_t)err));
}

namespace {

inline size_t up16(size_t x) { return (x + 15) & ~(size_t)15; }

// Exact row-store / record sizes of a static-band job; worst case for adaptive.
void job_capacity(const HostWindow& w, int qlen, bool adaptive, int f, int wband, int64_t& rs_cap,
                  int64_t& tb_cap, int& max_bn) {
    const int m = qlen + 1;
    rs_cap = 0;
    tb_cap = 0;
    max_bn = 0;
    for (int i = 0; i < w.n; i++) {
        int Bs, Be;
        if (adaptive) {
            Bs = 0;
            Be = m / BLK + 2;
        } else {
            band_static(f, w.hq[i], w.tq[i], m, wband, Bs, Be);
        }
        if (i == 0) Bs = 0;
        int bn = std::max(0, Be - Bs - 1);
        int d = i == 0 ? 0 : w.in_ptr[i + 1] - w.in_ptr[i];
        int bpc = d >= 2 ? 4 : 1;
        rs_cap += (int64_t)bn * 16;
        tb_cap += (int64_t)up16((size_t)bn * BLK * bpc);
        max_bn = std::max(max_bn, bn);
    }
    rs_cap += 16;
    tb_cap += 16;
}

template <int NT>
void launch_plain(int njobs, const DpArgs* d_jobs, cudaStream_t s) {
    k_plain<NT><<<njobs, NT, 0, s>>>(d_jobs);
}

// Shared memory for the static kernel's row ring (below the 227 KB a block
// may use, leaving part of the unified L1 for the read-only window arrays).
// The adaptive kernel keeps its rows in global memory: a shared-memory ring
// of a few full-width rows measured slower there (less L1 for the rest).
constexpr int kRingBytes = 160 * 1024;
constexpr int kRingMaxRows = 32;

template <int NT>
void launch_static(int njobs, const DpArgs* d_jobs, size_t dyn, cudaStream_t s) {
    if (dyn > 48 * 1024)
        cuda_check(cudaFuncSetAttribute(k_plain_static<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn),
                   "smem attr (k_plain_static)");
    k_plain_static<NT><<<njobs, NT, dyn, s>>>(d_jobs);
}

void launch_static_by_width(int max_bn, int njobs, const DpArgs* d_jobs, size_t dyn, cudaStream_t s) {
    if (max_bn <= 64) launch_static<64>(njobs, d_jobs, dyn, s);
    else if (max_bn <= 128) launch_static<128>(njobs, d_jobs, dyn, s);
    else if (max_bn <= 192) launch_static<192>(njobs, d_jobs, dyn, s);
    else if (max_bn <= 256) launch_static<256>(njobs, d_jobs, dyn, s);
    else if (max_bn <= 384) launch_static<384>(njobs, d_jobs, dyn, s);
    else launch_static<512>(njobs, d_jobs, dyn, s);
}

void launch_by_width(int max_bn, int njobs, const DpArgs* d_jobs, cudaStream_t s) {
    if (max_bn <= 32) launch_plain<32>(njobs, d_jobs, s);
    else if (max_bn <= 64) launch_plain<64>(njobs, d_jobs, s);
    else if (max_bn <= 128) launch_plain<128>(njobs, d_jobs, s);
    else if (max_bn <= 256) launch_plain<256>(njobs, d_jobs, s);
    else launch_plain<512>(njobs, d_jobs, s);
}

}  // namespace

GpuEngine::GpuEngine(int device) : device_(device) {
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    cudaStream_t s;
    cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    stream_ = s;
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "cudaEventCreate");
    cuda_check(cudaEventCreate(&e1), "cudaEventCreate");
    ev0_ = e0;
    ev1_ = e1;
}

GpuEngine::~GpuEngine() {
    cudaSetDevice(device_);
    if (dbuf_) cudaFree(dbuf_);
    if (hbuf_) cudaFreeHost(hbuf_);
    if (ev0_) cudaEventDestroy((cudaEvent_t)ev0_);
    if (ev1_) cudaEventDestroy((cudaEvent_t)ev1_);
    if (stream_) cudaStreamDestroy((cudaStream_t)stream_);
}

void GpuEngine::reserve_device(size_t bytes) {
    if (bytes <= dcap_) return;
    size_t cap = std::max(bytes, dcap_ * 2);
    if (dbuf_) cuda_check(cudaFree(dbuf_), "cudaFree");
    dbuf_ = nullptr;
    dcap_ = 0;
    cuda_check(cudaMalloc((void**)&dbuf_, cap), "cudaMalloc(arena)");
    dcap_ = cap;
}

void GpuEngine::reserve_host(size_t bytes) {
    if (bytes <= hcap_) return;
    size_t cap = std::max(bytes, hcap_ * 2);
    if (hbuf_) cuda_check(cudaFreeHost(hbuf_), "cudaFreeHost");
    hbuf_ = nullptr;
    hcap_ = 0;
    cuda_check(cudaMallocHost((void**)&hbuf_, cap), "cudaMallocHost(staging)");
    hcap_ = cap;
}

void GpuEngine::align_many(const std::vector<const HostWindow*>& wins, const std::vector<const uint8_t*>& qs,
                           const std::vector<int32_t>& qlens, const std::vector<int32_t>& abs, const Params& p,
                           std::vector<AlignOut>& outs) {
    const int J = (int)wins.size();
    outs.assign(J, AlignOut());
    if (J == 0) return;
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)stream_;
    const Scoring sc = scoring_of(p);

    struct Lay {
        size_t in_ptr, in_row, in_w, in_base, base, ind, hq, hq_loc, tq, out_ptr, out_row, qs;
        size_t meta, state, rs, tb, res;
        int64_t rs_cap, tb_cap;
        int32_t moves_cap;
        int w;
    };
    std::vector<Lay> L(J);
    size_t up = up16(sizeof(DpArgs) * J);
    int max_bn_all = 1;
    bool any_adaptive = false;
    for (int t = 0; t < J; t++) {
        const HostWindow& w = *wins[t];
        const int n = w.n, E = (int)w.in_row.size(), E2 = (int)w.out_row.size();
        Lay& l = L[t];
        const int m = qlens[t] + 1;
        l.w = p.b + (p.f ? m / p.f : 0);
        l.in_ptr = up; up += up16(4 * (size_t)(n + 1));
        l.in_row = up; up += up16(4 * (size_t)E);
        l.in_w = up; up += up16(4 * (size_t)E);
        l.in_base = up; up += up16((size_t)E);
        l.base = up; up += up16((size_t)n);
        l.ind = up; up += up16(4 * (size_t)n);
        l.hq = up; up += up16(4 * (size_t)n);
        l.hq_loc = up; up += up16(4 * (size_t)n);
        l.tq = up; up += up16(4 * (size_t)n);
        l.out_ptr = up; up += up16(4 * (size_t)(n + 1));
        l.out_row = up; up += up16(4 * (size_t)E2);
        l.qs = up; up += up16((size_t)qs_bytes(qlens[t]));
        const bool adaptive = p.f > 0 && abs[t];
        int max_bn;
        job_capacity(w, qlens[t], adaptive, p.f, l.w, l.rs_cap, l.tb_cap, max_bn);
        // the CTA covers the widest row in one chunk (up to 512 threads): an
        // adaptive row can widen to the full query (max_bn = m/8 + 2), and
        // idle threads cost less than extra chunks, each a serial scan step
        max_bn_all = std::max(max_bn_all, max_bn);
        any_adaptive = any_adaptive || adaptive;
        l.moves_cap = n + m + 8;
    }
    size_t res_begin = up;
    size_t pos = up;
    for (int t = 0; t < J; t++) {
        L[t].res = pos;
        pos += up16(16 + 4 * (size_t)L[t].moves_cap);
    }
    size_t res_end = pos;
    for (int t = 0; t < J; t++) {
        const int n = wins[t]->n;
        L[t].meta = pos; pos += up16(sizeof(RowMeta) * (size_t)n);
        L[t].state = pos; pos += up16(4 * (size_t)AB_NSTATE * n);
        L[t].rs = pos; pos += up16(4 * (size_t)L[t].rs_cap);
        L[t].tb = pos; pos += up16((size_t)L[t].tb_cap);
    }
    reserve_device(pos);
    reserve_host(res_end);

    // static bands only: k_plain_static with a shared-memory ring of recent rows
    int ring_rows = 0;
    if (!any_adaptive) {
        ring_rows = std::min(kRingMaxRows, kRingBytes / (max_bn_all * 64));
        if (ring_rows < 2) ring_rows = 0;
    }
    const int ring_blocks = max_bn_all;
    const size_t ring_bytes = (size_t)ring_rows * ring_blocks * 64;

    char* h = hbuf_;
    char* d = dbuf_;
    DpArgs* jobs = reinterpret_cast<DpArgs*>(h);
    for (int t = 0; t < J; t++) {
        const HostWindow& w = *wins[t];
        const Lay& l = L[t];
        auto cp = [&](size_t off, const void* src, size_t bytes) {
            if (bytes) std::memcpy(h + off, src, bytes);
        };
        cp(l.in_ptr, w.in_ptr.data(), 4 * (size_t)(w.n + 1));
        cp(l.in_row, w.in_row.data(), 4 * w.in_row.size());
        cp(l.in_w, w.in_w.data(), 4 * w.in_w.size());
        cp(l.in_base, w.in_base.data(), w.in_base.size());
        cp(l.base, w.base.data(), (size_t)w.n);
        cp(l.ind, w.ind.data(), 4 * (size_t)w.n);
        cp(l.hq, w.hq.data(), 4 * (size_t)w.n);
        cp(l.hq_loc, w.hq_loc.data(), 4 * (size_t)w.n);
        cp(l.tq, w.tq.data(), 4 * (size_t)w.n);
        cp(l.out_ptr, w.out_ptr.data(), 4 * (size_t)(w.n + 1));
        cp(l.out_row, w.out_row.data(), 4 * w.out_row.size());
        make_qs(qs[t], qlens[t], reinterpret_cast<uint8_t*>(h + l.qs));
        DpArgs a;
        std::memset(&a, 0, sizeof(a));
        a.v.n = w.n;
        a.v.in_ptr = reinterpret_cast<const int32_t*>(d + l.in_ptr);
        a.v.in_row = reinterpret_cast<const int32_t*>(d + l.in_row);
        a.v.in_w = reinterpret_cast<const int32_t*>(d + l.in_w);
        a.v.in_base = reinterpret_cast<const uint8_t*>(d + l.in_base);
        a.v.base = reinterpret_cast<const uint8_t*>(d + l.base);
        a.v.ind = reinterpret_cast<const int32_t*>(d + l.ind);
        a.v.hq = reinterpret_cast<const int32_t*>(d + l.hq);
        a.v.hq_loc = reinterpret_cast<const int32_t*>(d + l.hq_loc);
        a.v.tq = reinterpret_cast<const int32_t*>(d + l.tq);
        a.v.out_ptr = reinterpret_cast<const int32_t*>(d + l.out_ptr);
        a.v.out_row = reinterpret_cast<const int32_t*>(d + l.out_row);
        a.qs = reinterpret_cast<const uint8_t*>(d + l.qs);
        a.qlen = qlens[t];
        a.ab_band = abs[t];
        a.f = p.f;
        a.w = l.w;
        a.sc = sc;
        a.meta = reinterpret_cast<RowMeta*>(d + l.meta);
        a.state = reinterpret_cast<int32_t*>(d + l.state);
        a.rs = reinterpret_cast<int32_t*>(d + l.rs);
        a.rs_cap = l.rs_cap;
        a.tb = reinterpret_cast<uint8_t*>(d + l.tb);
        a.tb_cap = l.tb_cap;
        a.ring_rows = ring_rows;
        a.ring_blocks = ring_rows > 0 ? ring_blocks : 0;
        a.out = reinterpret_cast<int32_t*>(d + l.res);
        a.moves = reinterpret_cast<int32_t*>(d + l.res + 16);
        a.moves_cap = l.moves_cap;
        jobs[t] = a;
    }
    cuda_check(cudaMemcpyAsync(d, h, res_begin, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync(H2D)");
    if (timing) cuda_check(cudaEventRecord((cudaEvent_t)ev0_, s), "cudaEventRecord");
    if (any_adaptive) launch_by_width(max_bn_all, J, reinterpret_cast<const DpArgs*>(d), s);
    else launch_static_by_width(max_bn_all, J, reinterpret_cast<const DpArgs*>(d), ring_bytes, s);
    cuda_check(cudaGetLastError(), "k_plain launch");
    if (timing) cuda_check(cudaEventRecord((cudaEvent_t)ev1_, s), "cudaEventRecord");
    cuda_check(cudaMemcpyAsync(h + res_begin, d + res_begin, res_end - res_begin, cudaMemcpyDeviceToHost, s),
               "cudaMemcpyAsync(D2H)");
    cuda_check(cudaStreamSynchronize(s), "DP kernel");
    stats.launches++;
    stats.alignments += J;
    stats.h2d_bytes += (int64_t)res_begin;
    stats.d2h_bytes += (int64_t)(res_end - res_begin);
    if (timing) {
        float ms = 0.f;
        cuda_check(cudaEventElapsedTime(&ms, (cudaEvent_t)ev0_, (cudaEvent_t)ev1_), "cudaEventElapsedTime");
        stats.kernel_ms += ms;
    }
    for (int t = 0; t < J; t++) {
        const int32_t* o = reinterpret_cast<const int32_t*>(h + L[t].res);
        AlignOut& r = outs[t];
        r.status = o[0];
        r.score = o[1];
        r.cells = o[3];
        stats.cells += o[3];
        if (r.status == ST_OK) {
            int nm = std::min(o[2], L[t].moves_cap);
            r.moves.assign(o + 4, o + 4 + nm);
        }
    }
}

}  // namespace pb
