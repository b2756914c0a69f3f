// Host driver of one wavefront engine (see hk_engine.h).
#include "hk_engine.h"

#include <algorithm>
#include <cstddef>
#include <cstring>

namespace hk {

namespace {
constexpr int kQueueArrays = 2 /*eq*/ + 2 /*idle*/ + kWfTypes /*sq*/ + 1 /*fq*/;
}  // namespace

size_t WfEngine::bytes_for(int capacity, int nemitters) {
    const size_t N = (size_t)capacity;
    const size_t shadow = N * (size_t)std::max(1, nemitters);
    return N * kSlotBytes + N * sizeof(int) * kQueueArrays + shadow * 16 * 3 + sizeof(WfCounters) +
           (sizeof(WfJob) + sizeof(unsigned long long)) * kWfMaxJobs + sizeof(WfSeg) * kWfMaxSegs;
}

WfEngine::WfEngine(const DevScene &S, int sm_count, const WfEngineConfig &cfg) : S_(S), cfg_(cfg) {
    if (cfg_.capacity < 1024 || cfg_.capacity > (1 << 26))
        throw HkError{HK_ERR_INVALID, "wavefront capacity must be in [1024, 2^26]"};
    for (int t : {cfg_.threads_extend, cfg_.threads_shade})
        if (t % 32 != 0 || t <= 0 || t > 256)
            throw HkError{HK_ERR_INVALID, "wavefront block sizes must be multiples of 32 up to 256"};
    const size_t N = (size_t)cfg_.capacity;
    W_.capacity = cfg_.capacity;
    W_.max_shadow = cfg_.capacity * std::max(1, S.nemitters);
    state_.alloc(N * kSlotBytes);
    queues_.alloc(N * sizeof(int) * kQueueArrays);
    shadow_.alloc((size_t)W_.max_shadow * 16 * 3);
    counters_.alloc(sizeof(WfCounters));
    jobs_.alloc(sizeof(WfJob) * kWfMaxJobs);
    finished_.alloc(sizeof(unsigned long long) * kWfMaxJobs);
    segs_.alloc(sizeof(WfSeg) * kWfMaxSegs);
    bytes_ = bytes_for(cfg_.capacity, S.nemitters);
    char *rec = state_.as<char>();   // slot records (kSlotBytes each, 256-byte aligned base)
    W_.ray_o.p = (float4 *)(rec + 0);
    W_.ray_d.p = (float4 *)(rec + 16);
    W_.beta.p = (float4 *)(rec + 32);
    W_.pix.p = (float4 *)(rec + 48);
    W_.rng.p = (uint4 *)(rec + 64);
    W_.hit.p = (float4 *)(rec + 80);
    W_.prev_wi.p = (float4 *)(rec + 96);
    W_.prev_wo.p = (float4 *)(rec + 112);
    W_.lacc.p = (float4 *)(rec + 128);
    W_.prev_pdf.p = (float *)(rec + 144);
    int *q = queues_.as<int>();
    W_.eq[0] = q; W_.eq[1] = q + N;
    W_.idle[0] = q + 2 * N; W_.idle[1] = q + 3 * N;
    for (int t = 0; t < kWfTypes; ++t) W_.sq[t] = q + (4 + t) * N;
    W_.fq = q + (4 + kWfTypes) * N;
    float4 *sh = shadow_.as<float4>();
    W_.sh_o = sh; W_.sh_d = sh + W_.max_shadow; W_.sh_c = sh + 2 * (size_t)W_.max_shadow;
    W_.ctr = counters_.as<WfCounters>();
    W_.jobs = jobs_.as<WfJob>();
    W_.segs = segs_.as<WfSeg>();
    h_ctr_.alloc(1);
    h_fin_.alloc(kWfMaxJobs);
    h_jobs_.alloc(kWfMaxJobs);
    h_segs_.alloc(kWfMaxSegs);
    h_head_.alloc(1);
    std::memset(h_ctr_.p, 0, sizeof(WfCounters));
    std::memset(h_fin_.p, 0, sizeof(unsigned long long) * kWfMaxJobs);
    int least = 0, greatest = 0;
    HK_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    HK_CUDA(cudaStreamCreateWithPriority(&streams_[0], cudaStreamNonBlocking, least));
    HK_CUDA(cudaStreamCreateWithPriority(&streams_[1], cudaStreamNonBlocking, greatest));
    stream_ = streams_[0];
    HK_CUDA(cudaEventCreateWithFlags(&ev_switch_, cudaEventDisableTiming));
    HK_CUDA(cudaEventCreateWithFlags(&ev_done_, cudaEventDisableTiming));
    HK_CUDA(cudaEventCreateWithFlags(&ev_plan_, cudaEventDisableTiming));
    // launch configuration: persistent grids of one wave of resident blocks
    L_.threads_extend = cfg_.threads_extend;
    L_.threads_shade = cfg_.threads_shade;
    L_.threads_shadow = cfg_.threads_extend;
    L_.threads_regen = 256;
    L_.lean_extend = cfg_.reg_lean & 1;
    L_.lean_shadow = (cfg_.reg_lean >> 1) & 1;
    L_.lean_shade = (cfg_.reg_lean >> 2) & 1;
    L_.shadow_tests = cfg_.shadow_tests >= 0 && cfg_.shadow_tests <= 2 ? cfg_.shadow_tests : 0;
    L_.closest_tests = cfg_.closest_tests == 2 ? 2 : 0;
    auto grid = [&](int which, int threads) {
        const bool lean = which == 0 ? L_.lean_extend : (which == 2 ? L_.lean_shadow : (which == 1 ? L_.lean_shade : false));
        const bool shared = (which == 2 && L_.shadow_tests == 2) || (which == 0 && L_.closest_tests == 2);
        return std::max(1, sm_count * std::max(1, wf_occupancy(which, threads, S.accel, lean, shared)));
    };
    L_.blocks_extend = grid(0, L_.threads_extend);
    L_.blocks_shade = grid(1, L_.threads_shade);
    L_.blocks_shadow = grid(2, L_.threads_shadow);
    L_.blocks_regen = grid(3, L_.threads_regen);
    L_.fetch_steps = cfg_.fetch_steps > 0 ? cfg_.fetch_steps : (S.accel == kAccelBvh8 ? 3 : 8);
    L_.fetch_min_idle = std::max(1, std::min(32, cfg_.fetch_min_idle));
    L_.fetch_steps_shadow = cfg_.fetch_steps_shadow > 0 ? cfg_.fetch_steps_shadow : L_.fetch_steps;
    L_.fetch_min_idle_shadow = cfg_.fetch_min_idle_shadow > 0 ? std::min(32, cfg_.fetch_min_idle_shadow)
                                                              : L_.fetch_min_idle;
    HK_CUDA(cudaGetLastError());
    reset();
}

WfEngine::~WfEngine() {
    for (cudaStream_t s : streams_)
        if (s) cudaStreamSynchronize(s);
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    for (cudaEvent_t e : {ev_done_, ev_plan_, ev_switch_, pe_[0], pe_[1]})
        if (e) cudaEventDestroy(e);
    for (cudaStream_t s : streams_)
        if (s) cudaStreamDestroy(s);
}

void WfEngine::set_priority(bool high) {
    cudaStream_t target = streams_[high ? 1 : 0];
    if (target == stream_) return;
    HK_CUDA(cudaEventRecord(ev_switch_, stream_));
    HK_CUDA(cudaStreamWaitEvent(target, ev_switch_, 0));
    stream_ = target;
}

void WfEngine::reset() {
    set_plan({}, 0);
    HK_CUDA(wf_launch_init(W_, stream_));
}

void WfEngine::set_job(int slot, WfJob J) {
    if (slot < 0 || slot >= kWfMaxJobs) throw HkError{HK_ERR_INVALID, "job slot out of range"};
    // Each slot has its own staging entry; a slot is rewritten only after its
    // previous job ended, long after that job's copy ran.
    J.finished = finished_.as<unsigned long long>() + slot;
    h_jobs_.p[slot] = J;
    HK_CUDA(cudaMemcpyAsync(jobs_.as<WfJob>() + slot, h_jobs_.p + slot, sizeof(WfJob), cudaMemcpyHostToDevice, stream_));
    HK_CUDA(cudaMemsetAsync(finished_.as<unsigned long long>() + slot, 0, sizeof(unsigned long long), stream_));
}

void WfEngine::set_plan(const std::vector<WfSeg> &segs, uint64_t total) {
    if (segs.size() > (size_t)kWfMaxSegs) throw HkError{HK_ERR_INVALID, "dispatch plan has too many pieces"};
    HK_CUDA(cudaEventSynchronize(ev_plan_));   // the staging copies of the previous plan have run
    if (!segs.empty()) {
        std::memcpy(h_segs_.p, segs.data(), sizeof(WfSeg) * segs.size());
        HK_CUDA(cudaMemcpyAsync(segs_.p, h_segs_.p, sizeof(WfSeg) * segs.size(), cudaMemcpyHostToDevice, stream_));
    }
    WfCounters &h = *h_head_.p;
    h.next_work = 0;
    h.total_work = total;
    h.seg_count = (unsigned)segs.size();
    h.pad0 = 0;
    // the dispatch head: next_work, total_work, seg_count (first 20 bytes)
    HK_CUDA(cudaMemcpyAsync(W_.ctr, &h, offsetof(WfCounters, pad0), cudaMemcpyHostToDevice, stream_));
    HK_CUDA(cudaEventRecord(ev_plan_, stream_));
}

void WfEngine::capture() {
    HK_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    cudaError_t e0 = wf_launch_iteration(S_, W_, L_, 0, stream_);
    cudaError_t e1 = wf_launch_iteration(S_, W_, L_, 1, stream_);
    cudaError_t ec = cudaStreamEndCapture(stream_, &graph_);
    if (e0 != cudaSuccess || e1 != cudaSuccess || ec != cudaSuccess) {
        if (graph_) cudaGraphDestroy(graph_);
        graph_ = nullptr;
        throw HkError{HK_ERR_CUDA, "wavefront graph capture failed"};
    }
    HK_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
}

void WfEngine::run(int iterations, bool use_graph, float *kernel_ms, int32_t *kernel_launches) {
    iterations += iterations & 1;   // the queues ping-pong: whole pairs only
    if (kernel_ms) {
        if (!pe_[0]) {
            HK_CUDA(cudaEventCreate(&pe_[0]));
            HK_CUDA(cudaEventCreate(&pe_[1]));
        }
        const int phase_launches[4] = {2, 1, kWfTypes, 1};
        for (int k = 0; k < iterations; ++k)
            for (int ph = 0; ph < 4; ++ph) {
                HK_CUDA(cudaEventRecord(pe_[0], stream_));
                HK_CUDA(wf_launch_phase(S_, W_, L_, k & 1, ph, stream_));
                HK_CUDA(cudaEventRecord(pe_[1], stream_));
                HK_CUDA(cudaEventSynchronize(pe_[1]));
                float ms = 0;
                HK_CUDA(cudaEventElapsedTime(&ms, pe_[0], pe_[1]));
                kernel_ms[ph] += ms;
                if (kernel_launches) kernel_launches[ph] += phase_launches[ph];
            }
        return;
    }
    if (!use_graph) {
        for (int k = 0; k < iterations; ++k) HK_CUDA(wf_launch_iteration(S_, W_, L_, k & 1, stream_));
        return;
    }
    if (!exec_) capture();
    for (int k = 0; k < iterations; k += 2) HK_CUDA(cudaGraphLaunch(exec_, stream_));
}

void WfEngine::fetch_status() {
    HK_CUDA(cudaMemcpyAsync(h_ctr_.p, W_.ctr, offsetof(WfCounters, log_n), cudaMemcpyDeviceToHost, stream_));
    HK_CUDA(cudaMemcpyAsync(h_fin_.p, finished_.p, sizeof(unsigned long long) * kWfMaxJobs, cudaMemcpyDeviceToHost,
                            stream_));
    HK_CUDA(cudaEventRecord(ev_done_, stream_));
}

void WfEngine::add_counters(unsigned long long *out_dev) { HK_CUDA(wf_launch_counters_add(W_, out_dev, stream_)); }

int WfEngine::launch_log(int which, uint32_t *rays, int max) {
    unsigned n = 0;
    HK_CUDA(cudaMemcpyAsync(&n, &W_.ctr->log_n[which], sizeof n, cudaMemcpyDeviceToHost, stream_));
    HK_CUDA(cudaStreamSynchronize(stream_));
    const int k = (int)std::min<unsigned>(n, (unsigned)std::min(max, kWfLaunchLog));
    if (k > 0) {
        HK_CUDA(cudaMemcpyAsync(rays, &W_.ctr->log_rays[which][0], sizeof(uint32_t) * k, cudaMemcpyDeviceToHost,
                                stream_));
        HK_CUDA(cudaStreamSynchronize(stream_));
    }
    return (int)n;
}

}  // namespace hk
