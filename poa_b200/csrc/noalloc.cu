// noalloc.cu - poa_align_noalloc: one poa() alignment on device-resident
// inputs that allocates nothing.
//
// Who needs it: callers that cannot allocate device memory at the time they
// align - code running inside a framework that owns the whole device pool,
// a service that forbids allocation on its request path to keep latency and
// memory use fixed, or a host that already placed the window in device
// memory and only wants the DP run on its own stream. cudaMalloc synchronises
// the device and can fail under memory pressure, so such callers need an
// entry point whose working memory exists before they call it.
//
// The working memory (row store, traceback records, row metadata, adaptive
// band state, shifted query) is the file-scope array below, a fixed
// POA_NOALLOC_SCRATCH_BYTES per GPU, held by every GPU that loads this
// library until the process exits. The entry point rejects a window whose
// worst-case need exceeds it (see poa_align_noalloc in include/poa_b200.h).
// Every call uses the same array and leaves its contents behind; the kernel
// writes every location before it reads it, so nothing has to be cleared
// between calls, but two calls whose kernels overlap on the GPU (different
// streams, or other host threads) race on it and must be serialised by the
// caller.
#include <cuda_runtime.h>

#include <atomic>
#include <climits>
#include <cstring>

#include "../../include/poa_b200.h"
#include "plain.cuh"

namespace pb {
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[POA_NOALLOC_SCRATCH_BYTES];

// Device address of the scratch array, per device. In host code the symbol
// g_noalloc_scratch is only a host-side stand-in, never a device address, so
// it is resolved with cudaGetSymbolAddress once per device (with that device
// current) on the first call there. The cache is atomic: first calls from
// several host threads may race to resolve it and store the same address.
// The address belongs to the device's context: a process that calls
// cudaDeviceReset on a device must not call poa_align_noalloc there again.
constexpr int kMaxDevices = 64;
static std::atomic<void*> g_scratch_addr[kMaxDevices];

int scratch_for_current_device(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return POA_CUDA;
    void* p = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!p) {
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return POA_CUDA;
        g_scratch_addr[dev].store(p, std::memory_order_release);
    }
    *out = p;
    return POA_OK;
}

inline size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

// The job descriptor travels as a kernel parameter (no device copy needed);
// the shifted query is built from the caller's encoded query in the scratch.
template <int NT>
__global__ void __launch_bounds__(NT, 1) k_plain_noalloc(DpArgs a, const uint8_t* __restrict__ q, uint8_t* qs) {
    const int64_t qsb = qs_bytes(a.qlen);
    for (int64_t x = threadIdx.x; x < qsb; x += NT) qs[x] = (x >= 2 && x < (int64_t)a.qlen + 2) ? q[x - 2] : 4;
    // score, move count and cells are only written on success: start them at 0
    if (threadIdx.x < 3) a.out[1 + threadIdx.x] = 0;
    __syncthreads();
    if (a.v.n <= 0) {
        if (threadIdx.x == 0) a.out[0] = ST_BAD_ARG;
        return;
    }
    constexpr int NW = NT / 32;
    __shared__ int4 s_sum[2 * NW];
    __shared__ unsigned long long s_key[NW];
    __shared__ RowShared sr[2];
    __shared__ int32_t s_upd[UPD_INTS];
    CtaGroup<NT> g{s_sum, s_key, sr, s_upd};
    dp_fill(g, a);
    __syncthreads();
    if (threadIdx.x == 0 && a.out[0] == ST_OK) {
        int32_t nm = 0;
        a.out[0] = backtrack_records(a, a.qlen + 1, nm);
        a.out[2] = nm;
    }
}

}  // namespace
}  // namespace pb

namespace {

// Worst-case scratch bytes of one window: every row at the full band width.
// Every term is computed in int64 from values checked to be non-negative, so
// no size can wrap; a window whose need exceeds `limit` stops the sum early.
int noalloc_need(int32_t n_rows, int32_t qlen, int32_t adaptive, int64_t limit, int64_t* bytes) {
    if (n_rows <= 0 || qlen < 0 || !bytes) return POA_BAD_ARG;
    const int64_t n = n_rows;
    const int64_t blocks = ((int64_t)qlen + 1) / pb::BLK + 1;  // widest possible row: the full band
    auto up = [](int64_t x) { return (x + 255) & ~(int64_t)255; };
    int64_t need = up(pb::qs_bytes(qlen));
    if (need > limit) { *bytes = need; return POA_OK; }
    need += up((int64_t)sizeof(pb::RowMeta) * n);
    if (adaptive) need += up(4 * (int64_t)pb::AB_NSTATE * n);
    if (need > limit) { *bytes = need; return POA_OK; }
    // blocks <= 2^28 and n < 2^31, so each product below stays under 2^63
    need += up(4 * (n * blocks * 16 + 16));                 // row store
    if (need > limit) { *bytes = need; return POA_OK; }
    need += up(n * (blocks * pb::BLK * 4 + 16) + 16);       // records
    *bytes = need;
    return need < 0 ? POA_BAD_ARG : POA_OK;
}

}  // namespace

extern "C" int poa_align_noalloc(const poa_dev_window* w, const uint8_t* q_dev, int32_t qlen, const poa_params* p,
                                 int32_t ab_band, int32_t* moves_dev, int32_t moves_cap, int32_t* result_dev,
                                 void* stream) {
    using namespace pb;
    if (!w || !p || (!q_dev && qlen > 0) || qlen < 0 || !moves_dev || !result_dev || w->n_rows <= 0)
        return POA_BAD_ARG;
    if (!w->in_ptr || !w->in_row || !w->in_weight || !w->in_base || !w->base || !w->ind || !w->hq || !w->hq_loc ||
        !w->tq || !w->out_ptr || !w->out_row)
        return POA_BAD_ARG;
    if ((int64_t)moves_cap < (int64_t)w->n_rows + (int64_t)qlen + 1) return POA_BAD_ARG;
    const bool adaptive = p->band_f > 0 && ab_band;
    int64_t need = 0;
    if (noalloc_need(w->n_rows, qlen, adaptive, (int64_t)POA_NOALLOC_SCRATCH_BYTES, &need) != POA_OK)
        return POA_BAD_ARG;
    if (need > (int64_t)POA_NOALLOC_SCRATCH_BYTES) return POA_OOM;  // window too large for the fixed scratch
    void* base = nullptr;
    if (scratch_for_current_device(&base) != POA_OK) return POA_CUDA;

    const int n = w->n_rows, m = qlen + 1;
    const int64_t blocks = (int64_t)m / BLK + 1;
    char* s = (char*)base;
    size_t o = 0;
    uint8_t* qs = (uint8_t*)(s + o); o += up256((size_t)qs_bytes(qlen));
    RowMeta* meta = (RowMeta*)(s + o); o += up256(sizeof(RowMeta) * (size_t)n);
    int32_t* state = (int32_t*)(s + o); if (adaptive) o += up256(4 * (size_t)AB_NSTATE * n);
    int32_t* rs = (int32_t*)(s + o);
    const int64_t rs_cap = (int64_t)n * blocks * 16 + 16;
    o += up256(4 * (size_t)rs_cap);
    uint8_t* tb = (uint8_t*)(s + o);
    const int64_t tb_cap = (int64_t)n * (blocks * BLK * 4 + 16) + 16;

    poa_params pn = *p;
    if (pn.mismatch > 0) pn.mismatch = -pn.mismatch;  // initPara sign rules, src/handle_input.cpp:45-51
    if (pn.gap_open > 0) pn.gap_open = -pn.gap_open;
    if (pn.gap_ext > 0) pn.gap_ext = -pn.gap_ext;
    DpArgs a;
    std::memset(&a, 0, sizeof(a));
    a.v = WinView{n, w->in_ptr, w->in_row, w->in_weight, w->in_base, w->base, w->ind,
                  w->hq, w->hq_loc, w->tq, w->out_ptr, w->out_row};
    a.qs = qs;
    a.qlen = qlen;
    a.ab_band = ab_band;
    a.f = pn.band_f;
    a.w = pn.band_b + (pn.band_f ? m / pn.band_f : 0);
    a.sc.match = pn.match;
    a.sc.mismatch = pn.mismatch;
    a.sc.e1 = pn.gap_ext;
    a.sc.o1 = pn.gap_open + pn.gap_ext;
    a.meta = meta;
    a.state = state;
    a.rs = rs;
    a.rs_cap = rs_cap;
    a.ring_rows = 0;
    a.ring_blocks = 0;
    a.tb = tb;
    a.tb_cap = tb_cap;
    a.moves = moves_dev;
    a.moves_cap = moves_cap;
    a.out = result_dev;
    cudaStream_t st = (cudaStream_t)stream;
    k_plain_noalloc<128><<<1, 128, 0, st>>>(a, q_dev, qs);
    return cudaGetLastError() == cudaSuccess ? POA_OK : POA_CUDA;
}
