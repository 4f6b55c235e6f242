// proposer.cu - features, network (training and inference) and window plan of
// the learned band proposer; see proposer.h for what it predicts and why.
//
// Everything here is hand-written CUDA: a tiled BF16 x BF16 -> FP32 GEMM for
// the convolutions (as im2col products) and the dense layers, small
// elementwise kernels for im2col / col2im, ReLU masks, pooling, the loss and
// Adam, the minimizer feature kernel and the plan kernel.
#include "proposer.h"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <stdexcept>

#include "batch.h"
#include "gpu_engine.h"
#include "sketch.h"

namespace pb {
namespace {

typedef __nv_bfloat16 bf16;

constexpr int T = PROP_BINS;
constexpr int KC1 = PROP_KW * PROP_CIN;  // im2col width of layer 1
constexpr int KC = PROP_KW * PROP_CH;    // im2col width of layers 2, 3
// parameter offsets (floats)
constexpr int OW1 = 0, OB1 = OW1 + PROP_CH * KC1;
constexpr int OW2 = OB1 + PROP_CH, OB2 = OW2 + PROP_CH * KC;
constexpr int OW3 = OB2 + PROP_CH, OB3 = OW3 + PROP_CH * KC;
constexpr int OW4 = OB3 + PROP_CH, OB4 = OW4 + PROP_CH * PROP_CH;
constexpr int OW5 = OB4 + PROP_CH, OB5 = OW5 + PROP_OUT * PROP_CH;
static_assert(OB5 + PROP_OUT == PROP_NPARAM, "parameter layout");
// extras
constexpr int X_MEAN = 0, X_STD = 4, X_NODE_MARGIN = 8, X_TB_MARGIN = 9, X_SPILL_PER_ROW = 10, X_SPILL_MIN = 11;

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

// ---------------------------------------------------------------------------
// GEMM: C[M][N] = A x B (+ bias[n]) (ReLU), FP32 accumulation of BF16 operands.
// A element (m,k) = TA ? A[k*lda + m] : A[m*lda + k];
// B element (k,n) = TB ? B[n*ldb + k] : B[k*ldb + n].
// 64x64 tile per CTA of 256 threads (4x4 outputs each), K in steps of 16.
constexpr int GT = 64, GK = 16;

template <bool TA, bool TB>
__global__ void __launch_bounds__(256) k_gemm(const bf16* __restrict__ A, int lda, const bf16* __restrict__ B, int ldb,
                                              float* __restrict__ C, bf16* __restrict__ Cb, int ldc, int64_t M, int N,
                                              int64_t K, const float* __restrict__ bias, int relu) {
    __shared__ float As[GK][GT + 4];
    __shared__ float Bs[GK][GT + 4];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int64_t m0 = (int64_t)blockIdx.x * GT;
    const int n0 = blockIdx.y * GT;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
    for (int64_t k0 = 0; k0 < K; k0 += GK) {
        for (int e = tid; e < GT * GK; e += 256) {
            int mm, kk;
            if (TA) { mm = e % GT; kk = e / GT; } else { kk = e % GK; mm = e / GK; }
            const int64_t gm = m0 + mm, gk = k0 + kk;
            float v = 0.f;
            if (gm < M && gk < K) v = __bfloat162float(TA ? A[gk * lda + gm] : A[gm * lda + gk]);
            As[kk][mm] = v;
        }
        for (int e = tid; e < GT * GK; e += 256) {
            int nn, kk;
            if (TB) { kk = e % GK; nn = e / GK; } else { nn = e % GT; kk = e / GT; }
            const int gn = n0 + nn;
            const int64_t gk = k0 + kk;
            float v = 0.f;
            if (gn < N && gk < K) v = __bfloat162float(TB ? B[(int64_t)gn * ldb + gk] : B[gk * ldb + gn]);
            Bs[kk][nn] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int64_t gm = m0 + ty * 4 + i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int gn = n0 + tx * 4 + j;
            if (gn >= N) continue;
            float v = acc[i][j];
            if (bias) v += bias[gn];
            if (relu) v = fmaxf(v, 0.f);
            if (C) C[gm * ldc + gn] = v;
            if (Cb) Cb[gm * ldc + gn] = __float2bfloat16(v);
        }
    }
}

template <bool TA, bool TB>
void gemm(cudaStream_t s, const bf16* A, int lda, const bf16* B, int ldb, float* C, bf16* Cb, int ldc, int64_t M,
          int N, int64_t K, const float* bias, int relu) {
    if (M <= 0 || N <= 0) return;
    dim3 grid((unsigned)cdiv(M, GT), (unsigned)cdiv(N, GT));
    k_gemm<TA, TB><<<grid, 256, 0, s>>>(A, lda, B, ldb, C, Cb, ldc, M, N, K, bias, relu);
}

// ---------------------------------------------------------------------------
// elementwise kernels (grid-stride)
#define GRID_STRIDE(i, n) for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

inline unsigned grid_of(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, 256), 148 * 16)); }

// Xc[r][k*C + c] = x[r + k - 1][c] when bin t + k - 1 of the same read is in range
__global__ void k_im2col(const bf16* __restrict__ x, bf16* __restrict__ xc, int64_t rows, int C) {
    const int KCw = PROP_KW * C;
    GRID_STRIDE(i, rows * KCw) {
        const int c = (int)(i % C);
        const int k = (int)((i / C) % PROP_KW);
        const int64_t r = i / KCw;
        const int tt = (int)(r % T) + k - 1;
        xc[i] = (tt >= 0 && tt < T) ? x[(r + k - 1) * C + c] : __float2bfloat16(0.f);
    }
}

// dy[r][c] = (sum_k dxc[r - k + 1][k*C + c]) * (y[r][c] > 0), as BF16
__global__ void k_col2im_relu(const float* __restrict__ dxc, const bf16* __restrict__ y, bf16* __restrict__ dy,
                              int64_t rows, int C) {
    const int KCw = PROP_KW * C;
    GRID_STRIDE(i, rows * C) {
        const int c = (int)(i % C);
        const int64_t r = i / C;
        const int t = (int)(r % T);
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < PROP_KW; k++) {
            const int tt = t - k + 1;
            if (tt >= 0 && tt < T) s += dxc[(r - k + 1) * KCw + k * C + c];
        }
        dy[i] = __float2bfloat16(__bfloat162float(y[i]) > 0.f ? s : 0.f);
    }
}

// h[b][c] = mean over bins of y[b*T + t][c]
__global__ void k_pool(const bf16* __restrict__ y, bf16* __restrict__ h, int64_t nb) {
    GRID_STRIDE(i, nb * PROP_CH) {
        const int c = (int)(i % PROP_CH);
        const int64_t b = i / PROP_CH;
        float s = 0.f;
        for (int t = 0; t < T; t++) s += __bfloat162float(y[(b * T + t) * PROP_CH + c]);
        h[i] = __float2bfloat16(s * (1.f / T));
    }
}

// dy[b*T + t][c] = dh[b][c] / T * (y > 0)
__global__ void k_unpool_relu(const float* __restrict__ dh, const bf16* __restrict__ y, bf16* __restrict__ dy,
                              int64_t nb) {
    GRID_STRIDE(i, nb * T * PROP_CH) {
        const int c = (int)(i % PROP_CH);
        const int64_t b = i / ((int64_t)T * PROP_CH);
        const float g = dh[b * PROP_CH + c] * (1.f / T);
        dy[i] = __float2bfloat16(__bfloat162float(y[i]) > 0.f ? g : 0.f);
    }
}

// out = d * (y > 0) as BF16
__global__ void k_relu_mask(const float* __restrict__ d, const bf16* __restrict__ y, bf16* __restrict__ out, int64_t n) {
    GRID_STRIDE(i, n) out[i] = __float2bfloat16(__bfloat162float(y[i]) > 0.f ? d[i] : 0.f);
}

__global__ void k_to_bf16(const float* __restrict__ x, bf16* __restrict__ y, int64_t n) {
    GRID_STRIDE(i, n) y[i] = __float2bfloat16(x[i]);
}

// training batch: rows idx[0..nb) of X (host layout [n][T][CIN]) and of the
// standardised targets
__global__ void k_gather(const float* __restrict__ X, const float* __restrict__ Y, const int32_t* __restrict__ idx,
                         int nb, const float* __restrict__ extra, bf16* __restrict__ xb, float* __restrict__ yb) {
    GRID_STRIDE(i, (int64_t)nb * T * PROP_CIN) {
        const int64_t b = i / (T * PROP_CIN);
        xb[i] = __float2bfloat16(X[(int64_t)idx[b] * T * PROP_CIN + i % (T * PROP_CIN)]);
    }
    GRID_STRIDE(i, (int64_t)nb * PROP_OUT) {
        const int64_t b = i / PROP_OUT;
        const int o = (int)(i % PROP_OUT);
        yb[i] = (Y[(int64_t)idx[b] * PROP_OUT + o] - extra[X_MEAN + o]) / extra[X_STD + o];
    }
}

// mean squared error over nb x 4 outputs; gradient as BF16; loss summed into *loss
__global__ void k_loss(const float* __restrict__ o, const float* __restrict__ y, bf16* __restrict__ dob, int nb,
                       float* __restrict__ loss) {
    __shared__ float red[256];
    float acc = 0.f;
    const float scale = 1.f / (float)(nb * PROP_OUT);
    for (int i = threadIdx.x; i < nb * PROP_OUT; i += blockDim.x) {
        const float d = o[i] - y[i];
        acc += d * d * scale;
        dob[i] = __float2bfloat16(2.f * d * scale);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss += red[0];
}

// g[n] = sum over rows of d[r][n]; one CTA per column
__global__ void k_colsum(const bf16* __restrict__ d, int64_t rows, int N, float* __restrict__ g) {
    __shared__ float red[256];
    const int n = blockIdx.x;
    float acc = 0.f;
    for (int64_t r = threadIdx.x; r < rows; r += blockDim.x) acc += __bfloat162float(d[r * N + n]);
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) g[n] = red[0];
}

// Adam on the FP32 master weights, refreshing the BF16 copy
__global__ void k_adam(float* __restrict__ w, bf16* __restrict__ wb, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
    GRID_STRIDE(i, n) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        wb[i] = __float2bfloat16(wi);
    }
}

// raw outputs: y * std + mean
__global__ void k_destd(const float* __restrict__ o, const float* __restrict__ extra, float* __restrict__ y, int64_t n) {
    GRID_STRIDE(i, n * PROP_OUT) {
        const int k = (int)(i % PROP_OUT);
        y[i] = o[i] * extra[X_STD + k] + extra[X_MEAN + k];
    }
}

// ---------------------------------------------------------------------------
// minimizer features: one CTA per window, a hash table per CTA in global memory
constexpr int FT_THREADS = 128;
constexpr int FT_TILE = 1024;      // k-mer end positions per tile
constexpr int FT_MAXW = 32;        // largest minimizer window supported
constexpr int FT_MAXK = 28;

__device__ __forceinline__ int nt4_dev2(uint8_t c) {
    switch (c | 0x20) {
        case 'a': return 0;
        case 'c': return 1;
        case 'g': return 2;
        case 't': return 3;
        default: return 4;
    }
}

__device__ __forceinline__ uint32_t mm_key(uint64_t h) {
    const uint32_t k = (uint32_t)(h ^ (h >> 32));
    return k ? k : 1u;
}

// For the tile [p0, p0 + FT_TILE) of a read: hashes of k-mers ending at
// p0 - (w-1) .. p0 + FT_TILE + w - 2 (UINT64_MAX where no valid k-mer ends),
// then a flag per tile position: the k-mer ending there is the minimum of a
// full window of w consecutive valid k-mers (src/minimizer.cpp:60-135 for
// reads without an ambiguous base; equal minima in a window are all kept).
__device__ void sketch_tile(const uint8_t* rd, int len, int p0, int k, int w, uint8_t* sb, uint64_t* sh, uint8_t* flag) {
    const int H = FT_TILE + 2 * (w - 1);
    const int q0 = p0 - (w - 1) - (k - 1);  // first base needed
    const int nb = H + k - 1;
    for (int i = threadIdx.x; i < nb; i += FT_THREADS) {
        const int q = q0 + i;
        sb[i] = (q >= 0 && q < len) ? (uint8_t)nt4_dev2(rd[q]) : 4;
    }
    __syncthreads();
    const uint64_t mask = (k >= 32) ? ~0ull : ((1ull << (2 * k)) - 1);
    for (int i = threadIdx.x; i < H; i += FT_THREADS) {
        const int p = p0 - (w - 1) + i;  // k-mer end position
        uint64_t h = UINT64_MAX;
        if (p >= k - 1 && p < len) {
            uint64_t code = 0;
            bool ok = true;
            for (int j = 0; j < k; j++) {
                const int c = sb[i + j];
                ok &= c < 4;
                code = (code << 2) | (uint64_t)(c & 3);
            }
            if (ok) h = hash64(code & mask, mask);
        }
        sh[i] = h;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < FT_TILE; i += FT_THREADS) {
        const int c = i + (w - 1);  // index of the tile position in sh
        const uint64_t hp = sh[c];
        bool mn = false;
        if (hp != UINT64_MAX) {
            for (int s = c - (w - 1); s <= c && !mn; s++) {
                uint64_t wm = UINT64_MAX;
                bool full = true;
                for (int j = s; j < s + w; j++) {
                    full &= sh[j] != UINT64_MAX;
                    wm = sh[j] < wm ? sh[j] : wm;
                }
                mn = full && wm == hp;
            }
        }
        flag[i] = mn;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(FT_THREADS) k_features(const uint8_t* __restrict__ seq, const int64_t* __restrict__ read_off,
                                                        const int32_t* __restrict__ read_len,
                                                        const int32_t* __restrict__ win_off, int n_windows, int k, int w,
                                                        unsigned long long* __restrict__ tabs, int tab_bits,
                                                        float* __restrict__ X) {
    __shared__ uint8_t sb[FT_TILE + 2 * FT_MAXW + FT_MAXK];
    __shared__ uint64_t sh[FT_TILE + 2 * FT_MAXW];
    __shared__ uint8_t flag[FT_TILE];
    __shared__ float acc[T][3];
    const int tsize = 1 << tab_bits;
    unsigned long long* tab = tabs + (size_t)blockIdx.x * tsize;
    for (int win = blockIdx.x; win < n_windows; win += gridDim.x) {
        for (int i = threadIdx.x; i < tsize; i += FT_THREADS) tab[i] = 0ull;
        __syncthreads();
        const int r0 = win_off[win], r1 = win_off[win + 1];
        const int R = r1 - r0;
        // pass 1: count every minimizer of every read
        for (int r = r0; r < r1; r++) {
            const uint8_t* rd = seq + read_off[r];
            const int len = read_len[r];
            for (int p0 = 0; p0 < len; p0 += FT_TILE) {
                sketch_tile(rd, len, p0, k, w, sb, sh, flag);
                for (int i = threadIdx.x; i < FT_TILE; i += FT_THREADS) {
                    if (!flag[i]) continue;
                    const uint32_t key = mm_key(sh[i + w - 1]);
                    uint32_t slot = (key * 2654435761u) >> (32 - tab_bits);
                    for (int probe = 0; probe < tsize; probe++) {  // bounded: at most one pass over the table
                        unsigned long long cur = tab[slot];
                        if (cur == 0ull) {
                            cur = atomicCAS(&tab[slot], 0ull, ((unsigned long long)key << 32) | 1ull);
                            if (cur == 0ull) break;
                        }
                        if ((uint32_t)(cur >> 32) == key) {
                            atomicAdd(&tab[slot], 1ull);
                            break;
                        }
                        slot = (slot + 1) & (uint32_t)(tsize - 1);
                    }
                }
                __syncthreads();
            }
        }
        __syncthreads();
        // pass 2: per read and bin, density / anchored fraction / multiplicity
        const int L0 = R > 0 ? read_len[r0] : 0;
        for (int r = r0; r < r1; r++) {
            const uint8_t* rd = seq + read_off[r];
            const int len = read_len[r];
            for (int i = threadIdx.x; i < T * 3; i += FT_THREADS) (&acc[0][0])[i] = 0.f;
            __syncthreads();
            for (int p0 = 0; p0 < len; p0 += FT_TILE) {
                sketch_tile(rd, len, p0, k, w, sb, sh, flag);
                for (int i = threadIdx.x; i < FT_TILE; i += FT_THREADS) {
                    if (!flag[i]) continue;
                    const uint32_t key = mm_key(sh[i + w - 1]);
                    uint32_t slot = (key * 2654435761u) >> (32 - tab_bits);
                    int cnt = 0;
                    for (int probe = 0; probe < tsize; probe++) {
                        const unsigned long long cur = tab[slot];
                        if (cur == 0ull) break;
                        if ((uint32_t)(cur >> 32) == key) {
                            cnt = (int)(cur & 0xffffffffu);
                            break;
                        }
                        slot = (slot + 1) & (uint32_t)(tsize - 1);
                    }
                    const int others = max(cnt - 1, 0);
                    const int bin = (int)((int64_t)(p0 + i) * T / max(len, 1));
                    atomicAdd(&acc[bin][0], 1.f);
                    atomicAdd(&acc[bin][1], others > 0 ? 1.f : 0.f);
                    atomicAdd(&acc[bin][2], (float)min(others, max(R - 1, 1)));
                }
                __syncthreads();
            }
            for (int b = threadIdx.x; b < T; b += FT_THREADS) {
                const float blen = fmaxf((float)len / T, 1.f);
                const float nm = acc[b][0];
                float* x = X + ((int64_t)r * T + b) * PROP_CIN;
                x[0] = nm * (float)(w + 1) / (2.f * blen);
                x[1] = nm > 0.f ? acc[b][1] / nm : 0.f;
                x[2] = nm > 0.f ? 10.f * acc[b][2] / (nm * (float)max(R - 1, 1)) : 0.f;
                x[3] = (float)len / 2048.f;
                x[4] = (float)L0 / 2048.f;
                x[5] = (float)(r - r0) / 100.f;
                x[6] = (float)R / 100.f;
                x[7] = ((float)b + 0.5f) / T;
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// per-window plan from the per-read predictions (one thread per window)
__global__ void k_plan(const float* __restrict__ pred, const int32_t* __restrict__ read_len,
                       const int32_t* __restrict__ win_off, int n_windows, const float* __restrict__ extra,
                       int32_t* __restrict__ nodes_out, int64_t* __restrict__ tb_out, int64_t* __restrict__ spill_out,
                       float* __restrict__ cost_out) {
    GRID_STRIDE(wi, n_windows) {
        const int w = (int)wi;
        const int r0 = win_off[w], r1 = win_off[w + 1];
        double nodes = r1 > r0 ? 2.0 + read_len[r0] : 2.0;
        double maxtb = 0.0, maxrows = 0.0, cost = 0.0;
        for (int r = r0 + 1; r < r1; r++) {
            const float* y = pred + (int64_t)r * PROP_OUT;
            const double rows = nodes;
            const double m = (double)read_len[r] + 1.0;
            const double cells = fmin(fmax((double)y[1], 0.01), 1.0) * rows * m;
            const double bpc = fmin(fmax((double)y[2], 1.0), 4.0);
            maxtb = fmax(maxtb, cells * bpc);
            maxrows = fmax(maxrows, rows);
            cost += cells;
            nodes += fmax((double)y[0], 0.0) * read_len[r];
        }
        nodes_out[w] = (int32_t)fmin(nodes * extra[X_NODE_MARGIN] + 64.0, 2.0e9);
        tb_out[w] = (int64_t)(maxtb * extra[X_TB_MARGIN]) + 4096;
        spill_out[w] = (int64_t)fmax((double)extra[X_SPILL_MIN], maxrows * extra[X_SPILL_PER_ROW]);
        cost_out[w] = (float)cost;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// activations of one forward/backward pass over nb reads
struct Act {
    bf16 *x0, *xc1, *y1, *xc2, *y2, *xc3, *y3, *h, *z, *dob, *dzb, *dy3, *dy2, *dy1;
    float *o, *yt, *dz, *dh, *dxc, *loss;
};

static size_t act_layout(int64_t nb, Act* a, char* base) {
    const int64_t R = nb * T;
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t r = o; o = up256(o + bytes); return base ? base + r : nullptr; };
    Act t;
    t.x0 = (bf16*)take(2 * R * PROP_CIN);
    t.xc1 = (bf16*)take(2 * R * KC1);
    t.y1 = (bf16*)take(2 * R * PROP_CH);
    t.xc2 = (bf16*)take(2 * R * KC);
    t.y2 = (bf16*)take(2 * R * PROP_CH);
    t.xc3 = (bf16*)take(2 * R * KC);
    t.y3 = (bf16*)take(2 * R * PROP_CH);
    t.h = (bf16*)take(2 * nb * PROP_CH);
    t.z = (bf16*)take(2 * nb * PROP_CH);
    t.o = (float*)take(4 * nb * PROP_OUT);
    t.yt = (float*)take(4 * nb * PROP_OUT);
    t.dob = (bf16*)take(2 * nb * PROP_OUT);
    t.dz = (float*)take(4 * nb * PROP_CH);
    t.dzb = (bf16*)take(2 * nb * PROP_CH);
    t.dh = (float*)take(4 * nb * PROP_CH);
    t.dy3 = (bf16*)take(2 * R * PROP_CH);
    t.dxc = (float*)take(4 * R * KC);
    t.dy2 = (bf16*)take(2 * R * PROP_CH);
    t.dy1 = (bf16*)take(2 * R * PROP_CH);
    t.loss = (float*)take(64);
    if (a) *a = t;
    return o;
}

Proposer::Proposer(int device) : device_(device) {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    host_w_.assign(PROP_NWEIGHTS, 0.f);
    cuda_check(cudaMalloc(&d_w_, 4 * (size_t)PROP_NPARAM), "cudaMalloc(proposer)");
    cuda_check(cudaMalloc(&d_wb_, 2 * (size_t)PROP_NPARAM), "cudaMalloc(proposer)");
    cuda_check(cudaMalloc(&d_g_, 4 * (size_t)PROP_NPARAM), "cudaMalloc(proposer)");
    cuda_check(cudaMalloc(&d_m_, 4 * (size_t)PROP_NPARAM), "cudaMalloc(proposer)");
    cuda_check(cudaMalloc(&d_v_, 4 * (size_t)PROP_NPARAM), "cudaMalloc(proposer)");
    cuda_check(cudaMalloc(&d_extra_, 4 * (size_t)PROP_NEXTRA), "cudaMalloc(proposer)");
    // default initialisation: He-uniform weights from a fixed seed, zero biases,
    // identity standardisation, unit margins
    std::mt19937_64 rng(12345);
    auto init = [&](int off, int fan_out, int fan_in) {
        const float lim = std::sqrt(6.f / (float)fan_in);
        std::uniform_real_distribution<float> u(-lim, lim);
        for (int i = 0; i < fan_out * fan_in; i++) host_w_[off + i] = u(rng);
    };
    init(OW1, PROP_CH, KC1);
    init(OW2, PROP_CH, KC);
    init(OW3, PROP_CH, KC);
    init(OW4, PROP_CH, PROP_CH);
    init(OW5, PROP_OUT, PROP_CH);
    for (int k = 0; k < PROP_OUT; k++) host_w_[PROP_NPARAM + X_STD + k] = 1.f;
    host_w_[PROP_NPARAM + X_NODE_MARGIN] = 1.f;
    host_w_[PROP_NPARAM + X_TB_MARGIN] = 1.f;
    host_w_[PROP_NPARAM + X_SPILL_PER_ROW] = 8.f;
    host_w_[PROP_NPARAM + X_SPILL_MIN] = 65536.f;
    set_weights(host_w_.data());
}

Proposer::~Proposer() {
    cudaSetDevice(device_);
    if (graph_exec_) cudaGraphExecDestroy((cudaGraphExec_t)graph_exec_);
    for (void* p : {(void*)d_w_, (void*)d_wb_, (void*)d_g_, (void*)d_m_, (void*)d_v_, (void*)d_extra_, d_act_, d_tab_,
                    d_plan_, (void*)d_feat_, (void*)d_pred_})
        if (p) cudaFree(p);
}

void Proposer::upload_bf16(void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    k_to_bf16<<<grid_of(PROP_NPARAM), 256, 0, s>>>(d_w_, (bf16*)d_wb_, PROP_NPARAM);
    cuda_check(cudaGetLastError(), "k_to_bf16");
}

void Proposer::set_weights(const float* w) {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    std::memcpy(host_w_.data(), w, 4 * (size_t)PROP_NWEIGHTS);
    for (int k = 0; k < PROP_OUT; k++)
        if (!(host_w_[PROP_NPARAM + X_STD + k] > 0.f)) throw std::invalid_argument("proposer: output std must be > 0");
    cuda_check(cudaMemcpy(d_w_, host_w_.data(), 4 * (size_t)PROP_NPARAM, cudaMemcpyHostToDevice), "H2D weights");
    cuda_check(cudaMemcpy(d_extra_, host_w_.data() + PROP_NPARAM, 4 * (size_t)PROP_NEXTRA, cudaMemcpyHostToDevice),
               "H2D extras");
    cuda_check(cudaMemset(d_m_, 0, 4 * (size_t)PROP_NPARAM), "memset");
    cuda_check(cudaMemset(d_v_, 0, 4 * (size_t)PROP_NPARAM), "memset");
    upload_bf16(nullptr);
    cuda_check(cudaDeviceSynchronize(), "set_weights");
}

void Proposer::get_weights(float* w) const {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    std::vector<float> h(PROP_NPARAM);
    cuda_check(cudaMemcpy(h.data(), d_w_, 4 * (size_t)PROP_NPARAM, cudaMemcpyDeviceToHost), "D2H weights");
    std::memcpy(w, h.data(), 4 * (size_t)PROP_NPARAM);
    std::memcpy(w + PROP_NPARAM, host_w_.data() + PROP_NPARAM, 4 * (size_t)PROP_NEXTRA);
}

void Proposer::ensure(int64_t nb) {
    if (nb <= cap_) return;
    if (d_act_) cuda_check(cudaFree(d_act_), "cudaFree");
    d_act_ = nullptr;
    act_bytes_ = act_layout(nb, nullptr, nullptr);
    cuda_check(cudaMalloc(&d_act_, act_bytes_), "cudaMalloc(proposer activations)");
    cap_ = nb;
}

// forward over nb reads whose BF16 inputs are in act.x0; outputs (standardised) in act.o
void Proposer::forward(const float*, int64_t nb, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    Act a;
    act_layout(cap_, &a, (char*)d_act_);
    const bf16* W = (const bf16*)d_wb_;
    const int64_t R = nb * T;
    k_im2col<<<grid_of(R * KC1), 256, 0, s>>>(a.x0, a.xc1, R, PROP_CIN);
    gemm<false, true>(s, a.xc1, KC1, W + OW1, KC1, nullptr, a.y1, PROP_CH, R, PROP_CH, KC1, d_w_ + OB1, 1);
    k_im2col<<<grid_of(R * KC), 256, 0, s>>>(a.y1, a.xc2, R, PROP_CH);
    gemm<false, true>(s, a.xc2, KC, W + OW2, KC, nullptr, a.y2, PROP_CH, R, PROP_CH, KC, d_w_ + OB2, 1);
    k_im2col<<<grid_of(R * KC), 256, 0, s>>>(a.y2, a.xc3, R, PROP_CH);
    gemm<false, true>(s, a.xc3, KC, W + OW3, KC, nullptr, a.y3, PROP_CH, R, PROP_CH, KC, d_w_ + OB3, 1);
    k_pool<<<grid_of(nb * PROP_CH), 256, 0, s>>>(a.y3, a.h, nb);
    gemm<false, true>(s, a.h, PROP_CH, W + OW4, PROP_CH, nullptr, a.z, PROP_CH, nb, PROP_CH, PROP_CH, d_w_ + OB4, 1);
    gemm<false, true>(s, a.z, PROP_CH, W + OW5, PROP_CH, a.o, nullptr, PROP_OUT, nb, PROP_OUT, PROP_CH, d_w_ + OB5, 0);
    cuda_check(cudaGetLastError(), "proposer forward");
}

float Proposer::train(const float* X, const float* Y, int64_t n, int epochs, int batch, float lr, uint64_t seed,
                      float* losses) {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    if (n <= 0 || batch <= 0 || epochs <= 0) throw std::invalid_argument("proposer: empty training set");
    // standardisation of the targets from the training set
    for (int k = 0; k < PROP_OUT; k++) {
        double s = 0.0, s2 = 0.0;
        for (int64_t i = 0; i < n; i++) {
            s += Y[i * PROP_OUT + k];
            s2 += (double)Y[i * PROP_OUT + k] * Y[i * PROP_OUT + k];
        }
        const double mean = s / n, var = std::max(s2 / n - mean * mean, 1e-12);
        host_w_[PROP_NPARAM + X_MEAN + k] = (float)mean;
        host_w_[PROP_NPARAM + X_STD + k] = (float)std::sqrt(var);
    }
    cuda_check(cudaMemcpy(d_extra_, host_w_.data() + PROP_NPARAM, 4 * (size_t)PROP_NEXTRA, cudaMemcpyHostToDevice),
               "H2D extras");
    cudaStream_t s = nullptr;
    float *dX = nullptr, *dY = nullptr;
    int32_t* dIdx = nullptr;
    cuda_check(cudaMalloc(&dX, 4 * (size_t)n * T * PROP_CIN), "cudaMalloc(train X)");
    cuda_check(cudaMalloc(&dY, 4 * (size_t)n * PROP_OUT), "cudaMalloc(train Y)");
    cuda_check(cudaMalloc(&dIdx, 4 * (size_t)n), "cudaMalloc(train idx)");
    cuda_check(cudaMemcpy(dX, X, 4 * (size_t)n * T * PROP_CIN, cudaMemcpyHostToDevice), "H2D X");
    cuda_check(cudaMemcpy(dY, Y, 4 * (size_t)n * PROP_OUT, cudaMemcpyHostToDevice), "H2D Y");
    ensure(batch);
    Act a;
    act_layout(cap_, &a, (char*)d_act_);
    std::vector<int32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::mt19937_64 rng(seed);
    int step = 0;
    float last = 0.f;
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(idx.begin(), idx.end(), rng);
        cuda_check(cudaMemcpy(dIdx, idx.data(), 4 * (size_t)n, cudaMemcpyHostToDevice), "H2D idx");
        cuda_check(cudaMemset(a.loss, 0, 4), "memset loss");
        int nbatches = 0;
        for (int64_t b0 = 0; b0 < n; b0 += batch) {
            const int nb = (int)std::min<int64_t>(batch, n - b0);
            k_gather<<<grid_of((int64_t)nb * T * PROP_CIN), 256, 0, s>>>(dX, dY, dIdx + b0, nb, d_extra_, a.x0, a.yt);
            loss_and_gradient(nb, s);
            step++;
            const float b1 = 0.9f, b2 = 0.999f;
            k_adam<<<grid_of(PROP_NPARAM), 256, 0, s>>>(d_w_, (bf16*)d_wb_, d_g_, d_m_, d_v_, PROP_NPARAM, lr, b1, b2,
                                                        1e-8f, 1.f - std::pow(b1, (float)step),
                                                        1.f - std::pow(b2, (float)step));
            cuda_check(cudaGetLastError(), "proposer train step");
            nbatches++;
        }
        float lsum = 0.f;
        cuda_check(cudaMemcpy(&lsum, a.loss, 4, cudaMemcpyDeviceToHost), "D2H loss");
        last = lsum / (float)std::max(nbatches, 1);
        if (losses) losses[ep] = last;
    }
    cudaFree(dX);
    cudaFree(dY);
    cudaFree(dIdx);
    return last;
}

// Loss and parameter gradient of one batch whose BF16 inputs are in act.x0 and
// standardised targets in act.yt: forward, MSE (summed into act.loss), then
// the backward GEMMs, col2im / unpooling with the ReLU masks and the bias
// column sums into d_g_.
void Proposer::loss_and_gradient(int nb, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    Act a;
    act_layout(cap_, &a, (char*)d_act_);
    const bf16* W = (const bf16*)d_wb_;
    const int64_t R = (int64_t)nb * T;
    forward(nullptr, nb, s);
    k_loss<<<1, 256, 0, s>>>(a.o, a.yt, a.dob, nb, a.loss);
    // output layer
    gemm<true, false>(s, a.dob, PROP_OUT, a.z, PROP_CH, d_g_ + OW5, nullptr, PROP_CH, PROP_OUT, PROP_CH, nb,
                      nullptr, 0);
    k_colsum<<<PROP_OUT, 256, 0, s>>>(a.dob, nb, PROP_OUT, d_g_ + OB5);
    gemm<false, false>(s, a.dob, PROP_OUT, W + OW5, PROP_CH, a.dz, nullptr, PROP_CH, nb, PROP_CH, PROP_OUT,
                       nullptr, 0);
    k_relu_mask<<<grid_of((int64_t)nb * PROP_CH), 256, 0, s>>>(a.dz, a.z, a.dzb, (int64_t)nb * PROP_CH);
    // hidden dense layer
    gemm<true, false>(s, a.dzb, PROP_CH, a.h, PROP_CH, d_g_ + OW4, nullptr, PROP_CH, PROP_CH, PROP_CH, nb,
                      nullptr, 0);
    k_colsum<<<PROP_CH, 256, 0, s>>>(a.dzb, nb, PROP_CH, d_g_ + OB4);
    gemm<false, false>(s, a.dzb, PROP_CH, W + OW4, PROP_CH, a.dh, nullptr, PROP_CH, nb, PROP_CH, PROP_CH,
                       nullptr, 0);
    k_unpool_relu<<<grid_of(R * PROP_CH), 256, 0, s>>>(a.dh, a.y3, a.dy3, nb);
    // conv 3
    gemm<true, false>(s, a.dy3, PROP_CH, a.xc3, KC, d_g_ + OW3, nullptr, KC, PROP_CH, KC, R, nullptr, 0);
    k_colsum<<<PROP_CH, 256, 0, s>>>(a.dy3, R, PROP_CH, d_g_ + OB3);
    gemm<false, false>(s, a.dy3, PROP_CH, W + OW3, KC, a.dxc, nullptr, KC, R, KC, PROP_CH, nullptr, 0);
    k_col2im_relu<<<grid_of(R * PROP_CH), 256, 0, s>>>(a.dxc, a.y2, a.dy2, R, PROP_CH);
    // conv 2
    gemm<true, false>(s, a.dy2, PROP_CH, a.xc2, KC, d_g_ + OW2, nullptr, KC, PROP_CH, KC, R, nullptr, 0);
    k_colsum<<<PROP_CH, 256, 0, s>>>(a.dy2, R, PROP_CH, d_g_ + OB2);
    gemm<false, false>(s, a.dy2, PROP_CH, W + OW2, KC, a.dxc, nullptr, KC, R, KC, PROP_CH, nullptr, 0);
    k_col2im_relu<<<grid_of(R * PROP_CH), 256, 0, s>>>(a.dxc, a.y1, a.dy1, R, PROP_CH);
    // conv 1 (no input gradient)
    gemm<true, false>(s, a.dy1, PROP_CH, a.xc1, KC1, d_g_ + OW1, nullptr, KC1, PROP_CH, KC1, R, nullptr, 0);
    k_colsum<<<PROP_CH, 256, 0, s>>>(a.dy1, R, PROP_CH, d_g_ + OB1);
    cuda_check(cudaGetLastError(), "proposer backward");
}

float Proposer::gradient(const float* X, const float* Y, int64_t n, float* grad) {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    if (n <= 0 || n > 4096) throw std::invalid_argument("proposer: gradient batch must hold 1..4096 reads");
    float *dX = nullptr, *dY = nullptr;
    int32_t* dIdx = nullptr;
    cuda_check(cudaMalloc(&dX, 4 * (size_t)n * T * PROP_CIN), "cudaMalloc(grad X)");
    cuda_check(cudaMalloc(&dY, 4 * (size_t)n * PROP_OUT), "cudaMalloc(grad Y)");
    cuda_check(cudaMalloc(&dIdx, 4 * (size_t)n), "cudaMalloc(grad idx)");
    std::vector<int32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    cuda_check(cudaMemcpy(dX, X, 4 * (size_t)n * T * PROP_CIN, cudaMemcpyHostToDevice), "H2D X");
    cuda_check(cudaMemcpy(dY, Y, 4 * (size_t)n * PROP_OUT, cudaMemcpyHostToDevice), "H2D Y");
    cuda_check(cudaMemcpy(dIdx, idx.data(), 4 * (size_t)n, cudaMemcpyHostToDevice), "H2D idx");
    ensure(n);
    Act a;
    act_layout(cap_, &a, (char*)d_act_);
    cuda_check(cudaMemset(a.loss, 0, 4), "memset loss");
    k_gather<<<grid_of(n * T * PROP_CIN), 256>>>(dX, dY, dIdx, (int)n, d_extra_, a.x0, a.yt);
    loss_and_gradient((int)n, nullptr);
    float loss = 0.f;
    cuda_check(cudaMemcpy(grad, d_g_, 4 * (size_t)PROP_NPARAM, cudaMemcpyDeviceToHost), "D2H grad");
    cuda_check(cudaMemcpy(&loss, a.loss, 4, cudaMemcpyDeviceToHost), "D2H loss");
    cudaFree(dX);
    cudaFree(dY);
    cudaFree(dIdx);
    return loss;
}

constexpr int64_t PREDICT_CHUNK = 4096;

void Proposer::predict_device(const float* dX, int64_t n, float* dY, void* stream) {
    ensure(std::min<int64_t>(std::max<int64_t>(n, 1), PREDICT_CHUNK));
    predict_launch(dX, n, dY, stream);
}

// the inference launches only (buffers already sized by ensure)
void Proposer::predict_launch(const float* dX, int64_t n, float* dY, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    Act a;
    act_layout(cap_, &a, (char*)d_act_);
    for (int64_t b0 = 0; b0 < n; b0 += cap_) {
        const int64_t nb = std::min<int64_t>(cap_, n - b0);
        k_to_bf16<<<grid_of(nb * T * PROP_CIN), 256, 0, s>>>(dX + b0 * T * PROP_CIN, a.x0, nb * T * PROP_CIN);
        forward(nullptr, nb, s);
        k_destd<<<grid_of(nb * PROP_OUT), 256, 0, s>>>(a.o, d_extra_, dY + b0 * PROP_OUT, nb);
    }
    cuda_check(cudaGetLastError(), "proposer predict");
}

void Proposer::predict_host(const float* X, int64_t n, float* Y) {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    float *dX = nullptr, *dY = nullptr;
    cuda_check(cudaMalloc(&dX, 4 * (size_t)std::max<int64_t>(n, 1) * T * PROP_CIN), "cudaMalloc(predict X)");
    cuda_check(cudaMalloc(&dY, 4 * (size_t)std::max<int64_t>(n, 1) * PROP_OUT), "cudaMalloc(predict Y)");
    cuda_check(cudaMemcpy(dX, X, 4 * (size_t)n * T * PROP_CIN, cudaMemcpyHostToDevice), "H2D X");
    predict_device(dX, n, dY, nullptr);
    cuda_check(cudaMemcpy(Y, dY, 4 * (size_t)n * PROP_OUT, cudaMemcpyDeviceToHost), "D2H Y");
    cudaFree(dX);
    cudaFree(dY);
}

void Proposer::features(const DeviceWindows& dw, int k, int w, float* dX, void* stream) {
    if (dw.n_windows <= 0) return;
    int bits = 0, grid = 0;
    features_prep(dw, k, w, bits, grid);
    features_launch(dw, k, w, bits, grid, dX, stream);
}

void Proposer::features_launch(const DeviceWindows& dw, int k, int w, int bits, int grid, float* dX, void* stream) {
    k_features<<<grid, FT_THREADS, 0, (cudaStream_t)stream>>>(dw.seq, dw.read_off, dw.read_len, dw.win_off,
                                                               dw.n_windows, k, w, (unsigned long long*)d_tab_, bits,
                                                               dX);
    cuda_check(cudaGetLastError(), "k_features");
}

// hash-table size and grid of the feature kernel; allocates its scratch
void Proposer::features_prep(const DeviceWindows& dw, int k, int w, int& bits_out, int& grid_out) {
    if (k < 1 || k > FT_MAXK || w < 1 || w > FT_MAXW) throw std::invalid_argument("proposer: k or w out of range");
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    // table: at least twice the window's possible minimizers, a power of two
    const double est = (double)dw.max_win_bases * 2.0 / (w + 1) * 1.5 + 1024.0;
    int bits = 10;
    while ((double)(1ll << bits) < 2.0 * est && bits < 24) bits++;
    int sms = 0;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_), "attr");
    int grid = std::min(dw.n_windows, sms * 4);
    size_t need = (size_t)grid << bits;
    need *= 8;
    // keep the scratch modest: fewer CTAs for very large windows
    while (need > ((size_t)1 << 31) && grid > sms) {
        grid = std::max(sms, grid / 2);
        need = ((size_t)grid << bits) * 8;
    }
    if (need > tab_bytes_) {
        if (d_tab_) cuda_check(cudaFree(d_tab_), "cudaFree");
        d_tab_ = nullptr;
        cuda_check(cudaMalloc(&d_tab_, need), "cudaMalloc(proposer tables)");
        tab_bytes_ = need;
    }
    bits_out = bits;
    grid_out = grid;
}

void Proposer::plan(const DeviceWindows& dw, int k, int w, std::vector<int32_t>& nodes, std::vector<int64_t>& tb,
                    std::vector<int64_t>& spill, std::vector<float>& cost) {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)dw.stream;
    const int64_t nr = std::max<int64_t>(dw.n_reads, 1);
    const size_t fb = 4 * (size_t)nr * T * PROP_CIN, pb = 4 * (size_t)nr * PROP_OUT;
    if (fb > feat_bytes_) {
        if (d_feat_) cuda_check(cudaFree(d_feat_), "cudaFree");
        d_feat_ = nullptr;
        cuda_check(cudaMalloc(&d_feat_, fb), "cudaMalloc(proposer features)");
        feat_bytes_ = fb;
    }
    if (pb > pred_bytes_) {
        if (d_pred_) cuda_check(cudaFree(d_pred_), "cudaFree");
        d_pred_ = nullptr;
        cuda_check(cudaMalloc(&d_pred_, pb), "cudaMalloc(proposer predictions)");
        pred_bytes_ = pb;
    }
    const int nw = dw.n_windows;
    const size_t need = up256(4 * (size_t)nw) + 3 * up256(8 * (size_t)nw);
    if (need > plan_bytes_) {
        if (d_plan_) cuda_check(cudaFree(d_plan_), "cudaFree");
        d_plan_ = nullptr;
        cuda_check(cudaMalloc(&d_plan_, need), "cudaMalloc(proposer plan)");
        plan_bytes_ = need;
    }
    nodes.assign(nw, 0);
    tb.assign(nw, 0);
    spill.assign(nw, 0);
    cost.assign(nw, 0.f);
    if (nw == 0) return;
    int bits = 0, grid = 0;
    features_prep(dw, k, w, bits, grid);
    ensure(std::min<int64_t>(std::max<int64_t>(dw.n_reads, 1), PREDICT_CHUNK));
    char* p = (char*)d_plan_;
    int32_t* dn = (int32_t*)p;
    int64_t* dt = (int64_t*)(p + up256(4 * (size_t)nw));
    int64_t* ds = (int64_t*)(p + up256(4 * (size_t)nw) + up256(8 * (size_t)nw));
    float* dc = (float*)(p + up256(4 * (size_t)nw) + 2 * up256(8 * (size_t)nw));
    // features, inference and plan: ~10 launches per 4,096 reads, recorded once as a
    // CUDA graph per batch shape and replayed with one launch
    const GraphKey key{dw.seq, dw.read_off, dw.read_len, dw.win_off, dw.n_reads, nw, k, w, bits, grid,
                       d_feat_, d_pred_, d_plan_, d_tab_, d_act_, cap_, s};
    if (!graph_exec_ || std::memcmp(&key, &graph_key_, sizeof key) != 0) {
        if (graph_exec_) cudaGraphExecDestroy((cudaGraphExec_t)graph_exec_);
        graph_exec_ = nullptr;
        cudaGraph_t gr = nullptr;
        cuda_check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
        try {
            features_launch(dw, k, w, bits, grid, d_feat_, s);
            predict_launch(d_feat_, dw.n_reads, d_pred_, s);
            k_plan<<<grid_of(nw), 256, 0, s>>>(d_pred_, dw.read_len, dw.win_off, nw, d_extra_, dn, dt, ds, dc);
            cuda_check(cudaGetLastError(), "k_plan");
        } catch (...) {
            cudaStreamEndCapture(s, &gr);
            if (gr) cudaGraphDestroy(gr);
            throw;
        }
        cuda_check(cudaStreamEndCapture(s, &gr), "end capture");
        cudaGraphExec_t ex = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&ex, gr, 0);
        cudaGraphDestroy(gr);
        cuda_check(e, "graph instantiate");
        graph_exec_ = ex;
        std::memcpy(&graph_key_, &key, sizeof key);
    }
    cuda_check(cudaGraphLaunch((cudaGraphExec_t)graph_exec_, s), "graph launch");
    cuda_check(cudaMemcpyAsync(nodes.data(), dn, 4 * (size_t)nw, cudaMemcpyDeviceToHost, s), "D2H plan");
    cuda_check(cudaMemcpyAsync(tb.data(), dt, 8 * (size_t)nw, cudaMemcpyDeviceToHost, s), "D2H plan");
    cuda_check(cudaMemcpyAsync(spill.data(), ds, 8 * (size_t)nw, cudaMemcpyDeviceToHost, s), "D2H plan");
    cuda_check(cudaMemcpyAsync(cost.data(), dc, 4 * (size_t)nw, cudaMemcpyDeviceToHost, s), "D2H plan");
    cuda_check(cudaStreamSynchronize(s), "proposer plan");
}

}  // namespace pb
