// proposer.h - the learned band proposer of the batched window engine.
//
// minipoa sizes nothing ahead of an alignment: poa() allocates its DP
// matrices per call (src/align.cpp:1397, full n x m with -B) and the graph
// grows with every fused read (src/graph.cpp:170-235). The batch engine runs
// a whole window in one fixed device slot, so it needs, before the launch,
// each window's graph size and the traceback bytes of its largest alignment.
// The proposer predicts them from minimizer features of the reads:
//
//   features  one CTA per window: the (w,k)-minimizers of every read
//             (src/minimizer.cpp:60-135 semantics, forward strand), counted in
//             a per-window hash table; per read and per position bin, the
//             minimizer density, the fraction of its minimizers that anchor to
//             another read of the window, and the mean anchor multiplicity,
//             plus read length, first-read length, read index and read count.
//   network   3 x Conv1d(k=3, 64 channels, ReLU) over 32 bins -> mean pool ->
//             Linear(64,64)+ReLU -> Linear(64,4). BF16 weights and activations
//             as GEMM operands, FP32 accumulation, FP32 master weights (Adam).
//   outputs   per read: new graph nodes per query base, mean band width as a
//             fraction of the query (band cells / (rows * m)), traceback bytes
//             per cell, mean band centre as a fraction of the query.
//   plan      per window, on the device: graph nodes after every read (a
//             prefix sum of the predicted growth), band cells and record bytes
//             of every alignment, their maximum, times the calibrated margins.
//
// The plan only sizes slots and orders windows; every DP still computes the
// reference's own band, so results do not depend on the proposer. A window
// whose alignment outgrows its slot is re-run with the default sizing.
#pragma once
#include <stdint.h>

#include <vector>

namespace pb {

constexpr int PROP_K = 15, PROP_W = 10;  // minimizer k-mer and window of the features
constexpr int PROP_BINS = 32;   // position bins along a read
constexpr int PROP_CIN = 8;     // input channels
constexpr int PROP_CH = 64;     // conv / hidden channels
constexpr int PROP_KW = 3;      // conv kernel width
constexpr int PROP_OUT = 4;     // outputs per read
// FP32 parameters: W1[64][3*8] b1 W2[64][3*64] b2 W3[64][3*64] b3 W4[64][64] b4 W5[4][64] b5
constexpr int PROP_NPARAM = PROP_CH * PROP_KW * PROP_CIN + PROP_CH + 2 * (PROP_CH * PROP_KW * PROP_CH + PROP_CH) +
                            PROP_CH * PROP_CH + PROP_CH + PROP_OUT * PROP_CH + PROP_OUT;
// after the parameters: output mean[4], output std[4], node margin, record-byte
// margin, spilled row-store entries per DP row, minimum spill entries
constexpr int PROP_NEXTRA = 12;
constexpr int PROP_NWEIGHTS = PROP_NPARAM + PROP_NEXTRA;

struct DeviceWindows;

class Proposer {
  public:
    explicit Proposer(int device);
    ~Proposer();
    Proposer(const Proposer&) = delete;
    Proposer& operator=(const Proposer&) = delete;

    // PROP_NWEIGHTS floats (parameters, then the extras above).
    void set_weights(const float* w);
    void get_weights(float* w) const;

    // Train on host arrays: X [n][PROP_BINS][PROP_CIN], Y [n][PROP_OUT] (raw
    // targets; standardised with the stored mean/std). Mini-batch Adam, the
    // sample order shuffled per epoch from `seed`. Returns the last epoch's
    // mean loss; per-epoch losses go to `losses` (may be null).
    float train(const float* X, const float* Y, int64_t n, int epochs, int batch, float lr, uint64_t seed,
                float* losses);
    // Loss (mean squared error on the standardised targets) and the gradient
    // of every parameter (PROP_NPARAM floats) for one batch of n <= 4096 reads,
    // without an update: the backward kernels the training step runs.
    float gradient(const float* X, const float* Y, int64_t n, float* grad);
    // Inference on host arrays: Y [n][PROP_OUT] raw (de-standardised) outputs.
    void predict_host(const float* X, int64_t n, float* Y);
    // Inference on device arrays (stream order on `stream`).
    void predict_device(const float* dX, int64_t n, float* dY, void* stream);

    // Features of every read of the uploaded windows, into device memory
    // (dX: n_reads * PROP_BINS * PROP_CIN floats).
    void features(const DeviceWindows& dw, int k, int w, float* dX, void* stream);
    // Features + inference + per-window plan on the device; the plan comes
    // back to the host (one value per window each).
    void plan(const DeviceWindows& dw, int k, int w, std::vector<int32_t>& nodes, std::vector<int64_t>& tb,
              std::vector<int64_t>& spill, std::vector<float>& cost);

    float extra(int i) const { return host_w_[PROP_NPARAM + i]; }

  private:
    // the plan's launches are replayed from a CUDA graph while these stay the same
    struct GraphKey {
        const void *seq, *read_off, *read_len, *win_off;
        int64_t n_reads;
        int32_t n_windows, k, w, bits, grid;
        const void *feat, *pred, *plan, *tab, *act;
        int64_t cap;
        const void* stream;
    };
    void features_prep(const DeviceWindows& dw, int k, int w, int& bits, int& grid);
    void features_launch(const DeviceWindows& dw, int k, int w, int bits, int grid, float* dX, void* stream);
    void predict_launch(const float* dX, int64_t n, float* dY, void* stream);
    void* graph_exec_ = nullptr;
    GraphKey graph_key_{};
    void ensure(int64_t batch_reads);
    void forward(const float* dX, int64_t n, void* stream);
    void loss_and_gradient(int nb, void* stream);
    void upload_bf16(void* stream);
    int device_;
    std::vector<float> host_w_;
    // device parameters
    float* d_w_ = nullptr;        // FP32 master
    uint16_t* d_wb_ = nullptr;    // BF16 copy (GEMM operands)
    float* d_g_ = nullptr;        // gradients
    float* d_m_ = nullptr;        // Adam first moment
    float* d_v_ = nullptr;        // Adam second moment
    float* d_extra_ = nullptr;    // the PROP_NEXTRA floats
    // activations for up to cap_ reads
    int64_t cap_ = 0;
    void* d_act_ = nullptr;
    size_t act_bytes_ = 0;
    // feature scratch: per-CTA hash tables
    void* d_tab_ = nullptr;
    size_t tab_bytes_ = 0;
    // plan scratch
    void* d_plan_ = nullptr;
    size_t plan_bytes_ = 0;
    float* d_feat_ = nullptr;
    size_t feat_bytes_ = 0;
    float* d_pred_ = nullptr;
    size_t pred_bytes_ = 0;
};

}  // namespace pb
