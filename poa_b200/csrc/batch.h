// batch.h - the batched window engine: thousands of independent POA windows
// (one read set -> one consensus each) in one persistent launch. Each warp
// owns a slot of device memory holding one window's graph and DP buffers
// and runs minipoa's whole per-window loop on the device: align the read
// (the same DP fill as the plain kernel, on a warp), fuse the path into the
// graph, re-sort it, next read; then the heaviest-path consensus.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "driver.h"

namespace pb {

struct BatchInput {
    const uint8_t* seq;       // all reads' ASCII bases back to back
    int64_t seq_bytes;
    const int64_t* read_off;  // [n_reads]
    const int32_t* read_len;  // [n_reads]
    int32_t n_reads;
    const int32_t* win_off;   // [n_windows + 1] read ranges per window
    int32_t n_windows;
};

constexpr int NRSTAT = 8;

class Proposer;

// Device copies of an uploaded batch (valid until the next upload).
struct DeviceWindows {
    const uint8_t* seq;
    const int64_t* read_off;
    const int32_t* read_len;
    const int32_t* win_off;
    int32_t n_reads, n_windows, max_len;
    int64_t max_win_bases;
    void* stream;
};

struct BatchStats {
    double kernel_ms = 0.0;   // device time of the last run()'s kernel launches (CUDA events)
    double run_ms = 0.0;      // device time of the whole last run(): plan, launches, re-runs
    double plan_ms = 0.0;     // device time of the proposer's plan inside run()
    int64_t cells = 0;        // DP band cells of the last run
    int64_t edge_cells = 0;   // band cells x in-window predecessors of their rows
    int64_t dp_calls = 0;
    int32_t slots = 0;        // concurrent windows (warps) of the persistent launch
    int64_t slot_bytes = 0;
    int64_t h2d_bytes = 0, d2h_bytes = 0;
    int32_t failed = 0;       // windows that ended with a non-OK status
    int32_t retried = 0;      // windows re-run with larger capacities
    int32_t fallback = 0;     // windows that outgrew the plan's sizing (re-run with the default sizing)
    int32_t launches = 0;     // kernel launches of the last run()
    // summed lane-0 clock cycles per phase over all windows: view build, DP
    // fill, backtrack, fusion, topological sort, consensus
    int64_t phase_cycles[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

class BatchEngine {
  public:
    explicit BatchEngine(int device);
    ~BatchEngine();
    // Copy the windows into device memory (kept resident for run()).
    void upload(const BatchInput& in, const Params& p);
    // Run every uploaded window on the device; device time lands in stats.
    void run();
    // Per-window consensus (ASCII) and status of the last run().
    void download(std::vector<std::string>& cons, std::vector<int32_t>& status);
    // Resource plan of the uploaded windows (a band proposer's prediction), one
    // value per window: graph nodes, traceback record bytes and spilled
    // row-store entries of its largest alignment, and a relative cost (the
    // windows run largest first). The plan sizes the slots only; every DP
    // still runs the reference's band, and a window that outgrows its slot is
    // re-run with the default sizing (counted in stats.fallback). nullptr
    // clears the plan. Cleared by upload().
    void set_plan(const int32_t* nodes, const int64_t* tb_bytes, const int64_t* spill, const float* cost);
    DeviceWindows device_windows() const;
    // Plan every run() with this proposer first (nullptr: no proposer).
    void set_proposer(Proposer* p) { proposer_ = p; }
    // Device-side totals only (no consensus copy): cells and failures.
    void sync_stats();
    // Per read of the last run(), NRSTAT values: [0] widest DP row in blocks,
    // [1] band cells, [2] DP rows, [3] graph nodes after fusing the read,
    // [4] traceback record bytes, [5] spilled row-store entries (int32),
    // [6] graph edges after fusing the read, [7] mean band centre (midpoint
    // column over the DP rows) in thousandths of the query length. A window's
    // first read has no DP ([0..2], [4], [5], [7] zero).
    void read_stats(std::vector<int32_t>& out);
    BatchStats stats;
    int32_t warps_per_block = 4;
    int32_t blocks_per_sm = 3;  // 3: 168-register build; >= 4: 128-register build (occupancy still caps it)
    int32_t smem_per_warp = 18432;  // shared-memory row ring + staging / topsort workspace per warp
    int32_t max_blocks = 0;         // cap on the persistent grid (0 = one wave of resident blocks)

  private:
    void ensure(void** ptr, size_t* cap, size_t bytes);
    struct Caps {
        int32_t NC;      // graph nodes per slot
        int64_t tb_cap;  // traceback record bytes
        int64_t spill;   // spilled row-store entries (int32)
    };
    Caps default_caps(int scale) const;
    int ring_blocks() const;
    // one persistent launch over `count` windows (ids) with slots of the given
    // capacities, grown by up to `headroom` when memory allows every resident warp one
    void launch(const int32_t* windows, int32_t count, const Caps& caps, double headroom = 1.0);
    static constexpr double PLAN_HEADROOM = 1.5;
    Proposer* proposer_ = nullptr;
    void* kgraph_exec_ = nullptr;      // the launch as a CUDA graph, and the launch it was recorded for
    std::vector<char> kgraph_key_;
    void* evr0_ = nullptr;
    void* evr1_ = nullptr;
    void* evp_ = nullptr;
  public:
    // the plan of the last planned run (empty when the run had none)
    const std::vector<int32_t>& plan_nodes() const { return plan_nodes_; }
    const std::vector<int64_t>& plan_tb() const { return plan_tb_; }
    const std::vector<int64_t>& plan_spill() const { return plan_spill_; }

  private:
    std::vector<int32_t> plan_nodes_, plan_order_;
    std::vector<int64_t> plan_tb_, plan_spill_;
    int device_;
    void* stream_ = nullptr;
    void* ev0_ = nullptr;
    void* ev1_ = nullptr;
    Params p_;
    int32_t n_windows_ = 0, n_reads_ = 0, max_len_ = 0, cons_stride_ = 0;
    int64_t max_win_bases_ = 0;
    // device buffers
    void* d_in_ = nullptr;      size_t d_in_cap_ = 0;    // reads + offsets + window table + order
    void* d_out_ = nullptr;     size_t d_out_cap_ = 0;   // consensus + lengths + status + cells
    void* d_slots_ = nullptr;   size_t d_slots_cap_ = 0;
    void* h_out_ = nullptr;     size_t h_out_cap_ = 0;   // pinned mirror of d_out_
    size_t off_seq_ = 0, off_roff_ = 0, off_rlen_ = 0, off_woff_ = 0, off_order_ = 0, off_ctr_ = 0;
    size_t out_cons_ = 0, out_len_ = 0, out_status_ = 0, out_cells_ = 0, out_phase_ = 0, out_rstats_ = 0, out_bytes_ = 0;
    std::vector<int32_t> order_;
};

}  // namespace pb
