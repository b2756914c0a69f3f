// Host driver of one wavefront engine: the path-slot pool of one scene in HBM,
// its job table and dispatch plan, its own stream and the CUDA graph of its
// iterations.  hk_render_batch runs one engine per scene over a fixed batch;
// the serving loop keeps one engine per resident scene and adds jobs to it
// while it runs.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "hk_device.h"
#include "hk_hostutil.h"
#include "hk_wavefront.h"

namespace hk {

struct WfEngineConfig {
    int capacity = 1 << 21;   // path slots
    int threads_extend = 128;
    int threads_shade = 128;
    int fetch_steps = 0;      // node visits between traversal refills (0: per-tree default)
    int fetch_min_idle = 1;   // idle lanes before a warp refills while others traverse
    int fetch_steps_shadow = 0;      // the same for the shadow rays (0: the closest-hit value)
    int fetch_min_idle_shadow = 0;
    int reg_lean = 0;   // bit 0: extend, bit 1: shadow, bit 2: untextured shade kernels with the smaller register budget
    int shadow_tests = 0;   // shadow rays' triangle tests: 0 per lane, 1 postponed, 2 shared over the warp
    int closest_tests = 0;  // closest-hit rays' triangle tests: 0 per lane, 2 shared over the warp
};

class WfEngine {
public:
    // S must stay valid (its device buffers alive) for the engine's lifetime.
    WfEngine(const DevScene &S, int sm_count, const WfEngineConfig &cfg);
    ~WfEngine();
    WfEngine(const WfEngine &) = delete;
    WfEngine &operator=(const WfEngine &) = delete;

    // Device bytes an engine of this capacity holds for a scene with nemitters emitters.
    static size_t bytes_for(int capacity, int nemitters);
    size_t device_bytes() const { return bytes_; }
    const WfEngineConfig &config() const { return cfg_; }
    // The stream the engine's work goes to next (one of two of different priority).
    cudaStream_t stream() const { return stream_; }
    // Move later work to the high- or low-priority stream, ordered after all
    // earlier work: pending kernels of a high-priority engine are scheduled
    // before those of low-priority engines sharing the GPU.
    void set_priority(bool high);

    // Empty pool (every slot idle), zero statistics, empty plan.  Async on stream().
    void reset();
    // Job-table entry `slot`: its finished counter is zeroed and J.finished set.  Async;
    // the slot must not be in use by paths in flight.
    void set_job(int slot, WfJob J);
    // Dispatch plan: pieces sorted by plan_begin, `total` items.  Async.
    void set_plan(const std::vector<WfSeg> &segs, uint64_t total);
    // `iterations` (even) wavefront iterations, from the graph or as plain launches.
    // With kernel_ms (host float[4]) each phase is timed with events and added.
    void run(int iterations, bool use_graph, float *kernel_ms = nullptr, int32_t *kernel_launches = nullptr);
    // Copy the counters and the job table's finished counters to the host mirrors
    // and record done_event(); read them after the event completed.
    void fetch_status();
    cudaEvent_t done_event() const { return ev_done_; }
    const WfCounters &status() const { return *h_ctr_.p; }
    const unsigned long long *finished() const { return h_fin_.p; }
    // Add the statistics to a caller's 7-slot device array.  Async.
    void add_counters(unsigned long long *out_dev);
    // Rays of each extend (which 0) / shadow (which 1) launch since the last
    // reset, in launch order: up to max of them into rays (host); returns the
    // number of launches.  Synchronises the engine's stream.
    int launch_log(int which, uint32_t *rays, int max);
    const WfState &state() const { return W_; }

private:
    void capture();
    DevScene S_;
    WfEngineConfig cfg_;
    WfLaunchConfig L_{};
    WfState W_{};
    size_t bytes_ = 0;
    DevBuf state_, queues_, shadow_, counters_, jobs_, finished_, segs_;
    PinnedBuf<WfCounters> h_ctr_;
    PinnedBuf<unsigned long long> h_fin_;
    PinnedBuf<WfJob> h_jobs_;
    PinnedBuf<WfSeg> h_segs_;
    PinnedBuf<WfCounters> h_head_;
    cudaStream_t stream_ = nullptr;             // current: streams_[0] or streams_[1]
    cudaStream_t streams_[2] = {nullptr, nullptr};   // low, high priority
    cudaEvent_t ev_switch_ = nullptr;
    cudaEvent_t ev_done_ = nullptr, ev_plan_ = nullptr, pe_[2] = {nullptr, nullptr};
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
};

}  // namespace hk
