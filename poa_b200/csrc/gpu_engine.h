// gpu_engine.h - runs poa() calls on the GPU: packs window views and queries
// into one pinned staging buffer, uploads it with a single copy, launches
// one CTA per alignment (plain.cuh) and reads back scores and moves.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "driver.h"

namespace pb {

struct EngineStats {
    int64_t launches = 0;      // kernel launches issued
    int64_t alignments = 0;    // poa() calls executed
    int64_t cells = 0;         // band cells computed (sum over rows of (Be-Bs-1)*8)
    double kernel_ms = 0.0;    // device time of the DP kernels (CUDA events)
    int64_t h2d_bytes = 0, d2h_bytes = 0;
};

class GpuEngine : public DpEngine {
  public:
    explicit GpuEngine(int device);
    ~GpuEngine() override;
    void align_many(const std::vector<const HostWindow*>& wins, const std::vector<const uint8_t*>& qs,
                    const std::vector<int32_t>& qlens, const std::vector<int32_t>& ab_bands, const Params& p,
                    std::vector<AlignOut>& outs) override;
    EngineStats stats;
    bool timing = false;  // record kernel time with CUDA events (adds a sync per call)

  private:
    void reserve_device(size_t bytes);
    void reserve_host(size_t bytes);
    int device_;
    void* stream_ = nullptr;
    void* ev0_ = nullptr;
    void* ev1_ = nullptr;
    char* dbuf_ = nullptr;
    size_t dcap_ = 0;
    char* hbuf_ = nullptr;
    size_t hcap_ = 0;
};

// Throws std::runtime_error with the CUDA message on failure.
void cuda_check(int err, const char* what);

}  // namespace pb
