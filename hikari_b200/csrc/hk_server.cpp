// Serving loop: continuous batching of render jobs over resident scenes.
//
// One host thread per server drives the device.  Each registered scene gets a
// wavefront engine (its path-slot pool, job table and stream) when its first
// job is admitted.  The thread repeats:
//   admit   queued jobs in arrival order while their film + image (and, for a
//           scene's first job, the pool) fit the device-memory budget and the
//           allocation succeeds; the job enters its scene's job table
//   launch  for every idle engine with work: a dispatch plan over its jobs'
//           undispensed work (least remaining first, or arrival order), then
//           `iterations_per_poll` wavefront iterations from the CUDA graph and
//           an async copy of the counters; when several scenes render, the one
//           with the least remaining job goes to its high-priority stream
//   poll    engines whose copy completed: the plan items consumed are credited
//           to their jobs; a job whose every item is dispensed and finished
//           is resolved and copied to its host buffer; a finished copy ends it
// Paths of new jobs enter the pool in the next iteration after admission, so
// jobs that arrive while others render share the pool with them.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/hikari_b200.h"
#include "hk_engine.h"
#include "hk_hostutil.h"
#include "hk_internal.h"
#include "hk_kernels.h"

using hk::guarded;
using hk::HkError;

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
    uint64_t id = 0;
    int scene = 0;
    hk_render_desc desc{};
    float *out = nullptr;
    bool out_pinned = false;
    hk::JobSize size{};
    uint64_t work = 0, dispensed = 0, paths = 0;
    uint64_t finished_seen = 0;  // work items finished at the last poll of its engine
    int state = HK_JOB_QUEUED;   // published state (under the server mutex)
    int phase = 0;               // server thread: 0 queued, 1 rendering, 2 copying out, 3 ended
    bool cancel = false;         // under the server mutex
    int slot = -1;
    void *film = nullptr, *rgb = nullptr;
    float *staging = nullptr;
    uint64_t bytes = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;
    cudaEvent_t ev = nullptr;
    // progressive preview (under the server mutex): a request names the host
    // buffer; the server thread resolves the film between iterations
    float *preview_dst = nullptr;
    int preview_state = 0;       // 0 none, 1 requested, 2 written
    double preview_fraction = 0.0;
};

struct SceneEntry {
    hk_scene *scene = nullptr;
    hk::SceneView view{};
    std::unique_ptr<hk::WfEngine> eng;
    std::vector<Job *> jobs;   // admitted and not ended
    std::vector<int> free_slots;
    bool inflight = false;
    std::vector<hk::WfSeg> plan;
    std::vector<Job *> plan_jobs;
    uint64_t plan_total = 0;
    unsigned long long rays = 0, shadow_rays = 0;
};

// Pinned staging buffers by size, reused across jobs.
struct PinnedCache {
    std::multimap<size_t, float *> free;
    float *get(size_t bytes) {
        auto it = free.find(bytes);
        if (it != free.end()) {
            float *p = it->second;
            free.erase(it);
            return p;
        }
        float *p = nullptr;
        HK_CUDA(cudaMallocHost((void **)&p, bytes));
        return p;
    }
    void put(float *p, size_t bytes) { free.emplace(bytes, p); }
    ~PinnedCache() {
        for (auto &kv : free) cudaFreeHost(kv.second);
    }
};

}  // namespace

struct hk_server {
    hk_server_config cfg{};
    hk::WfEngineConfig ec;
    int device = 0;
    Clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread th;
    bool stop = false;
    std::string fatal;
    std::vector<std::unique_ptr<SceneEntry>> scenes;           // under mu
    std::unordered_map<uint64_t, std::unique_ptr<Job>> jobs;   // under mu
    std::deque<Job *> incoming;                                 // under mu
    uint64_t next_id = 1;
    // statistics (under mu)
    uint64_t n_submitted = 0, n_done = 0, n_cancelled = 0, n_queued = 0, n_running = 0, paths_done = 0;
    unsigned long long rays = 0, shadow_rays = 0;
    double busy_s = 0;
    uint64_t in_use = 0, budget = 0;
    // server thread only
    std::deque<Job *> queued;
    std::vector<cudaEvent_t> event_pool;
    PinnedCache pinned;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
    void loop();
    void run_once(const std::vector<SceneEntry *> &sc, bool *progress);
    void admit(const std::vector<SceneEntry *> &sc);
    void launch(const std::vector<SceneEntry *> &sc);
    bool poll(const std::vector<SceneEntry *> &sc);
    void end_job(SceneEntry &e, Job *j, int state);
    void fail_all(const std::string &msg);
    void serve_previews(SceneEntry &e);
};

// Progressive preview (the headless stand-in for the reference's preview
// window, src/core/Screen.cpp): between iterations, when the scene's pool is
// idle, resolve each requested job's film as accumulated so far
// (ImageBlock::ToBitmap, src/core/Block.cpp:61) and copy it to the caller's
// buffer.
void hk_server::serve_previews(SceneEntry &e) {
    std::vector<Job *> want;
    {
        std::lock_guard<std::mutex> lk(mu);
        for (Job *j : e.jobs)
            if (j->phase == 1 && j->preview_state == 1) want.push_back(j);
    }
    if (want.empty()) return;
    cudaStream_t st = e.eng->stream();
    const unsigned long long *fin = e.eng->finished();
    for (Job *j : want) {
        HK_CUDA(hk::launch_resolve((const float *)j->film, (float *)j->rgb, (int)j->size.width, (int)j->size.height,
                                   e.view.dev->border, st));
        HK_CUDA(cudaMemcpyAsync(j->preview_dst, j->rgb, j->size.rgb_bytes, cudaMemcpyDeviceToHost, st));
    }
    HK_CUDA(cudaStreamSynchronize(st));
    {
        std::lock_guard<std::mutex> lk(mu);
        for (Job *j : want) {
            j->preview_fraction = j->work ? (double)fin[j->slot] / (double)j->work : 1.0;
            j->preview_state = 2;
        }
    }
    cv_done.notify_all();
}

void hk_server::end_job(SceneEntry &e, Job *j, int state) {
    if (e.eng) {
        cudaStream_t st = e.eng->stream();
        if (j->film) HK_CUDA(cudaFreeAsync(j->film, st));
        if (j->rgb) HK_CUDA(cudaFreeAsync(j->rgb, st));
    }
    j->film = j->rgb = nullptr;
    if (j->staging) pinned.put(j->staging, j->size.rgb_bytes);
    j->staging = nullptr;
    if (j->ev) event_pool.push_back(j->ev);
    j->ev = nullptr;
    if (j->slot >= 0) e.free_slots.push_back(j->slot);
    j->slot = -1;
    e.jobs.erase(std::remove(e.jobs.begin(), e.jobs.end(), j), e.jobs.end());
    j->phase = 3;
    std::lock_guard<std::mutex> lk(mu);
    in_use -= j->bytes;
    j->state = state;
    j->t_done = now();
    --n_running;
    if (state == HK_JOB_DONE) {
        ++n_done;
        paths_done += j->paths;
    } else {
        ++n_cancelled;
    }
    cv_done.notify_all();
}

void hk_server::admit(const std::vector<SceneEntry *> &sc) {
    {
        // queued jobs that were cancelled end now, wherever they are in the queue
        std::lock_guard<std::mutex> lk(mu);
        bool any = false;
        for (Job *j : queued)
            if (j->cancel) {
                j->state = HK_JOB_CANCELLED;
                j->t_done = now();
                j->phase = 3;
                --n_queued;
                ++n_cancelled;
                any = true;
            }
        if (any) {
            queued.erase(std::remove_if(queued.begin(), queued.end(), [](const Job *j) { return j->phase == 3; }),
                         queued.end());
            cv_done.notify_all();
        }
    }
    while (!queued.empty()) {
        Job *j = queued.front();
        SceneEntry &e = *sc[j->scene];
        const uint64_t need = j->size.film_bytes + j->size.rgb_bytes;
        const uint64_t pool = e.eng ? 0 : hk::WfEngine::bytes_for(ec.capacity, e.view.dev->nemitters);
        uint64_t used;
        {
            std::lock_guard<std::mutex> lk(mu);
            used = in_use;
        }
        if ((int)e.jobs.size() >= cfg.max_jobs || used + need + pool > budget) break;   // arrival order: wait
        if (!e.eng) {
            // the server's pool size and block sizes; the traversal knobs of
            // the scene's own configuration where it has one (autotuned)
            hk::WfEngineConfig sec = ec;
            if (*e.view.has_cfg) {
                const hk_wavefront_config &t = *e.view.cfg;
                sec.fetch_steps = std::max(0, std::min(1024, t.fetch_steps));
                sec.fetch_min_idle = t.fetch_min_idle > 0 ? std::min(32, t.fetch_min_idle) : 1;
                sec.fetch_steps_shadow = std::max(0, std::min(1024, t.fetch_steps_shadow));
                sec.fetch_min_idle_shadow = t.fetch_min_idle_shadow > 0 ? std::min(32, t.fetch_min_idle_shadow) : 0;
                sec.reg_lean = t.reg_lean & 7;
                sec.shadow_tests = t.shadow_tests >= 0 && t.shadow_tests <= 2 ? t.shadow_tests : 0;
                sec.closest_tests = t.closest_tests == 2 ? 2 : 0;
            }
            e.eng.reset(new hk::WfEngine(*e.view.dev, e.view.sm_count, sec));
            e.free_slots.clear();
            for (int k = cfg.max_jobs - 1; k >= 0; --k) e.free_slots.push_back(k);
            std::lock_guard<std::mutex> lk(mu);
            in_use += e.eng->device_bytes();
        }
        cudaStream_t st = e.eng->stream();
        if (cudaMallocAsync(&j->film, j->size.film_bytes, st) != cudaSuccess) {
            cudaGetLastError();
            j->film = nullptr;
            break;   // device memory is short right now: retry after jobs end
        }
        if (cudaMallocAsync(&j->rgb, j->size.rgb_bytes, st) != cudaSuccess) {
            cudaGetLastError();
            HK_CUDA(cudaFreeAsync(j->film, st));
            j->film = j->rgb = nullptr;
            break;
        }
        HK_CUDA(cudaMemsetAsync(j->film, 0, j->size.film_bytes, st));
        j->slot = e.free_slots.back();
        e.free_slots.pop_back();
        hk::WfJob J = hk::make_wf_job(e.scene, j->desc);
        J.film = (float *)j->film;
        e.eng->set_job(j->slot, J);
        j->bytes = need;
        j->phase = 1;
        e.jobs.push_back(j);
        queued.pop_front();
        std::lock_guard<std::mutex> lk(mu);
        in_use += need;
        j->state = HK_JOB_RUNNING;
        j->t_admit = now();
        --n_queued;
        ++n_running;
    }
}

void hk_server::launch(const std::vector<SceneEntry *> &sc) {
    // the scene holding the job with the least undispensed work (fully
    // dispensed jobs still rendering count as zero) runs at high priority
    const SceneEntry *urgent = nullptr;
    uint64_t least = UINT64_MAX;
    int busy = 0;
    // remaining work of each scene's least job: undispensed plus in flight
    // (work - finished), for the across-scenes gate
    std::vector<uint64_t> scene_least(sc.size(), UINT64_MAX);
    uint64_t global_least = UINT64_MAX;
    for (size_t k = 0; k < sc.size(); ++k) {
        SceneEntry *ep = sc[k];
        bool any = false;
        for (Job *j : ep->jobs)
            if (j->phase == 1) {
                any = true;
                const uint64_t rem = j->work - j->dispensed;
                if (rem < least) { least = rem; urgent = ep; }
                const uint64_t left = j->work - std::min<uint64_t>(j->finished_seen, j->work);
                scene_least[k] = std::min(scene_least[k], left);
            }
        busy += any ? 1 : 0;
        global_least = std::min(global_least, scene_least[k]);
    }
    for (size_t k = 0; k < sc.size(); ++k) {
        SceneEntry &e = *sc[k];
        if (!e.eng || e.inflight) continue;
        const bool gated = cfg.policy == HK_SERVE_SRPT_ACROSS ||
                           (cfg.policy == HK_SERVE_SRPT_SMALL && global_least <= cfg.small_work);
        if (gated && scene_least[k] != UINT64_MAX && scene_least[k] > (uint64_t)HK_SERVE_GATE * global_least)
            continue;   // waits while a much smaller job of another scene renders
        std::vector<Job *> rendering;
        for (Job *j : e.jobs)
            if (j->phase == 1) rendering.push_back(j);
        if (rendering.empty()) continue;
        std::vector<Job *> order;
        {
            std::lock_guard<std::mutex> lk(mu);
            for (Job *j : rendering)
                if (!j->cancel && j->dispensed < j->work) order.push_back(j);
        }
        if (cfg.policy == HK_SERVE_FIFO) {
            std::sort(order.begin(), order.end(), [](const Job *a, const Job *b) { return a->id < b->id; });
        } else {
            std::sort(order.begin(), order.end(), [](const Job *a, const Job *b) {
                uint64_t ra = a->work - a->dispensed, rb = b->work - b->dispensed;
                return ra != rb ? ra < rb : a->id < b->id;
            });
        }
        if (order.size() > (size_t)hk::kWfMaxSegs) order.resize(hk::kWfMaxSegs);
        e.plan.clear();
        e.plan_jobs.clear();
        uint64_t total = 0;
        for (Job *j : order) {
            e.plan.push_back(hk::WfSeg{total, j->dispensed, j->slot, 0});
            e.plan_jobs.push_back(j);
            total += j->work - j->dispensed;
        }
        e.plan_total = total;
        e.eng->set_priority(busy > 1 && &e == urgent);
        e.eng->set_plan(e.plan, total);
        e.eng->run(cfg.iterations_per_poll, true);
        e.eng->fetch_status();
        e.inflight = true;
    }
}

bool hk_server::poll(const std::vector<SceneEntry *> &sc) {
    bool progress = false;
    for (SceneEntry *ep : sc) {
        SceneEntry &e = *ep;
        if (!e.inflight && e.eng) serve_previews(e);
        if (e.inflight) {
            cudaError_t q = cudaEventQuery(e.eng->done_event());
            if (q == cudaErrorNotReady) continue;
            HK_CUDA(q);
            e.inflight = false;
            progress = true;
            const hk::WfCounters &h = e.eng->status();
            const uint64_t consumed = std::min<uint64_t>(h.next_work, e.plan_total);
            for (size_t k = 0; k < e.plan.size(); ++k) {
                const uint64_t b = e.plan[k].plan_begin;
                const uint64_t end = k + 1 < e.plan.size() ? e.plan[k + 1].plan_begin : e.plan_total;
                if (consumed > b) e.plan_jobs[k]->dispensed += std::min(end, consumed) - b;
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                rays += h.rays - e.rays;
                shadow_rays += h.shadow_rays - e.shadow_rays;
            }
            e.rays = h.rays;
            e.shadow_rays = h.shadow_rays;
            const unsigned long long *fin = e.eng->finished();
            std::vector<Job *> snapshot = e.jobs;
            for (Job *j : snapshot) {
                if (j->phase != 1) continue;
                const uint64_t f = fin[j->slot];
                j->finished_seen = f;
                bool cancel;
                {
                    std::lock_guard<std::mutex> lk(mu);
                    cancel = j->cancel;
                }
                if (cancel) {
                    if (f == j->dispensed) end_job(e, j, HK_JOB_CANCELLED);
                } else if (j->dispensed == j->work && f == j->work) {
                    cudaStream_t st = e.eng->stream();
                    HK_CUDA(hk::launch_resolve((const float *)j->film, (float *)j->rgb, (int)j->size.width,
                                               (int)j->size.height, e.view.dev->border, st));
                    float *dst = j->out;
                    if (!j->out_pinned) dst = j->staging = pinned.get(j->size.rgb_bytes);
                    HK_CUDA(cudaMemcpyAsync(dst, j->rgb, j->size.rgb_bytes, cudaMemcpyDeviceToHost, st));
                    if (event_pool.empty()) {
                        cudaEvent_t ev;
                        HK_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
                        event_pool.push_back(ev);
                    }
                    j->ev = event_pool.back();
                    event_pool.pop_back();
                    HK_CUDA(cudaEventRecord(j->ev, st));
                    j->phase = 2;
                }
            }
            serve_previews(e);   // the pool is idle until the next launch
        }
        std::vector<Job *> snapshot = e.jobs;
        for (Job *j : snapshot) {
            if (j->phase != 2) continue;
            cudaError_t q = cudaEventQuery(j->ev);
            if (q == cudaErrorNotReady) continue;
            HK_CUDA(q);
            if (j->staging) std::memcpy(j->out, j->staging, j->size.rgb_bytes);
            end_job(e, j, HK_JOB_DONE);
            progress = true;
        }
    }
    return progress;
}

void hk_server::fail_all(const std::string &msg) {
    std::lock_guard<std::mutex> lk(mu);
    fatal = msg;
    for (auto &kv : jobs) {
        Job *j = kv.second.get();
        if (j->state == HK_JOB_QUEUED || j->state == HK_JOB_RUNNING) {
            j->state = HK_JOB_FAILED;
            j->t_done = now();
        }
    }
    incoming.clear();
    queued.clear();
    cv_done.notify_all();
}

void hk_server::loop() {
    cudaSetDevice(device);
    double t_prev = now();
    try {
        for (;;) {
            std::vector<SceneEntry *> sc;
            bool any_running = false;
            {
                std::unique_lock<std::mutex> lk(mu);
                while (!incoming.empty()) {
                    queued.push_back(incoming.front());
                    incoming.pop_front();
                }
                for (auto &e : scenes) {
                    sc.push_back(e.get());
                    any_running = any_running || !e->jobs.empty();
                }
                const double t = now();
                if (n_running > 0) busy_s += t - t_prev;
                t_prev = t;
                if (queued.empty() && !any_running) {
                    if (stop) break;
                    cv_work.wait_for(lk, std::chrono::milliseconds(20));
                    t_prev = now();
                    continue;
                }
            }
            admit(sc);
            launch(sc);
            if (!poll(sc)) std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    } catch (const HkError &e) {
        fail_all(e.msg);
    } catch (const std::exception &e) {
        fail_all(e.what());
    }
}

namespace {

void status_of(const Job &j, hk_job_status *st) {
    std::memset(st, 0, sizeof *st);
    st->state = j.state;
    st->scene = j.scene;
    st->width = j.size.width;
    st->height = j.size.height;
    st->paths = j.paths;
    st->device_bytes = j.size.film_bytes + j.size.rgb_bytes;
    st->submit_s = j.t_submit;
    st->admit_s = j.t_admit;
    st->done_s = j.t_done;
    st->latency_s = j.state == HK_JOB_DONE ? j.t_done - j.t_submit : 0.0;
}

Job *find_job(hk_server *s, uint64_t id) {
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) throw HkError{HK_ERR_INVALID, "unknown job id"};
    return it->second.get();
}

}  // namespace

extern "C" {

int hk_server_create(const hk_server_config *cfg, hk_server **out) {
    return guarded([&] {
        if (!out) throw HkError{HK_ERR_INVALID, "null output pointer"};
        std::unique_ptr<hk_server> s(new hk_server());
        if (cfg) s->cfg = *cfg;
        hk_server_config &c = s->cfg;
        if (c.capacity <= 0) c.capacity = 1 << 19;   // small pools keep iterations short for newly admitted jobs
        if (c.threads_extend <= 0) c.threads_extend = 128;
        if (c.threads_shade <= 0) c.threads_shade = 128;
        if (c.iterations_per_poll <= 0) c.iterations_per_poll = 4;
        if (c.max_jobs <= 0) c.max_jobs = 256;
        if (c.small_work == 0) c.small_work = HK_SERVE_SMALL_WORK;
        if (c.max_jobs > hk::kWfMaxJobs) throw HkError{HK_ERR_INVALID, "max_jobs above 1024"};
        if (c.policy != HK_SERVE_SRPT && c.policy != HK_SERVE_FIFO && c.policy != HK_SERVE_SRPT_ACROSS &&
            c.policy != HK_SERVE_SRPT_SMALL)
            throw HkError{HK_ERR_INVALID, "unknown policy"};
        if (c.capacity < 1024 || c.capacity > (1 << 26)) throw HkError{HK_ERR_INVALID, "capacity outside [1024, 2^26]"};
        s->ec.capacity = c.capacity;
        s->ec.threads_extend = c.threads_extend;
        s->ec.threads_shade = c.threads_shade;
        HK_CUDA(cudaGetDevice(&s->device));
        size_t free_b = 0, total_b = 0;
        HK_CUDA(cudaMemGetInfo(&free_b, &total_b));
        s->budget = c.hbm_budget ? c.hbm_budget : (uint64_t)(0.9 * (double)free_b);
        // keep memory freed by ended jobs in the process's stream-ordered pool
        cudaMemPool_t pool;
        HK_CUDA(cudaDeviceGetDefaultMemPool(&pool, s->device));
        uint64_t keep = UINT64_MAX;
        HK_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        s->t0 = Clock::now();
        hk_server *raw = s.get();
        s->th = std::thread([raw] { raw->loop(); });
        *out = s.release();
        return HK_OK;
    });
}

int hk_server_destroy(hk_server *s) {
    return guarded([&] {
        if (!s) return HK_OK;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stop = true;
            for (auto &kv : s->jobs)
                if (kv.second->state == HK_JOB_QUEUED) kv.second->cancel = true;
        }
        s->cv_work.notify_all();
        if (s->th.joinable()) s->th.join();
        for (auto &e : s->scenes)
            if (e->eng) cudaStreamSynchronize(e->eng->stream());
        for (cudaEvent_t ev : s->event_pool) cudaEventDestroy(ev);
        delete s;
        return HK_OK;
    });
}

int hk_server_add_scene(hk_server *s, hk_scene *scene, int32_t *scene_id) {
    return guarded([&] {
        if (!s || !scene) throw HkError{HK_ERR_INVALID, "bad arguments"};
        std::unique_ptr<SceneEntry> e(new SceneEntry());
        e->scene = scene;
        e->view = hk::scene_view(scene);
        std::lock_guard<std::mutex> lk(s->mu);
        s->scenes.push_back(std::move(e));
        if (scene_id) *scene_id = (int32_t)s->scenes.size() - 1;
        return HK_OK;
    });
}

int hk_job_submit(hk_server *s, int32_t scene_id, const hk_render_desc *desc, float *rgb_host, uint64_t *job_id) {
    return guarded([&] {
        if (!s || !desc || !rgb_host) throw HkError{HK_ERR_INVALID, "bad arguments"};
        std::unique_ptr<Job> j(new Job());
        hk_scene *scene;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (!s->fatal.empty()) throw HkError{HK_ERR_CUDA, "server failed: " + s->fatal};
            if (scene_id < 0 || scene_id >= (int)s->scenes.size()) throw HkError{HK_ERR_INVALID, "unknown scene id"};
            scene = s->scenes[scene_id]->scene;
        }
        hk::WfJob J = hk::make_wf_job(scene, *desc);   // validates the request
        j->scene = scene_id;
        j->desc = *desc;
        j->out = rgb_host;
        j->size = hk::job_size(scene, *desc);
        j->work = J.work_count;
        j->paths = (uint64_t)j->size.width * j->size.height * (uint64_t)desc->spp;
        cudaPointerAttributes a{};
        if (cudaPointerGetAttributes(&a, rgb_host) == cudaSuccess) j->out_pinned = a.type == cudaMemoryTypeHost;
        else cudaGetLastError();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (j->size.film_bytes + j->size.rgb_bytes > s->budget)
                throw HkError{HK_ERR_NOMEM, "job needs more device memory than the server's budget"};
            j->id = s->next_id++;
            j->t_submit = s->now();
            if (job_id) *job_id = j->id;
            s->incoming.push_back(j.get());
            s->jobs[j->id] = std::move(j);
            ++s->n_submitted;
            ++s->n_queued;
        }
        s->cv_work.notify_all();
        return HK_OK;
    });
}

int hk_job_poll(hk_server *s, uint64_t id, hk_job_status *st) {
    return guarded([&] {
        if (!s || !st) throw HkError{HK_ERR_INVALID, "bad arguments"};
        std::lock_guard<std::mutex> lk(s->mu);
        status_of(*find_job(s, id), st);
        return HK_OK;
    });
}

int hk_job_wait(hk_server *s, uint64_t id, double timeout_s, hk_job_status *st) {
    return guarded([&] {
        if (!s) throw HkError{HK_ERR_INVALID, "bad arguments"};
        std::unique_lock<std::mutex> lk(s->mu);
        Job *j = find_job(s, id);
        auto ended = [&] { return j->state >= HK_JOB_DONE; };
        if (timeout_s < 0) s->cv_done.wait(lk, ended);
        else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ended)) {
            if (st) status_of(*j, st);
            throw HkError{HK_ERR_TIMEOUT, "job not finished within the timeout"};
        }
        if (st) status_of(*j, st);
        if (j->state == HK_JOB_FAILED) throw HkError{HK_ERR_CUDA, "server failed: " + s->fatal};
        return HK_OK;
    });
}

int hk_job_cancel(hk_server *s, uint64_t id) {
    return guarded([&] {
        if (!s) throw HkError{HK_ERR_INVALID, "bad arguments"};
        {
            std::lock_guard<std::mutex> lk(s->mu);
            find_job(s, id)->cancel = true;
        }
        s->cv_work.notify_all();
        return HK_OK;
    });
}

int hk_job_preview(hk_server *s, uint64_t id, float *rgb, double timeout_s, double *fraction) {
    return guarded([&] {
        if (!s || !rgb) throw HkError{HK_ERR_INVALID, "bad arguments"};
        std::unique_lock<std::mutex> lk(s->mu);
        Job *j = find_job(s, id);
        const size_t bytes = (size_t)j->size.width * j->size.height * 12;
        if (j->state == HK_JOB_QUEUED || j->state == HK_JOB_CANCELLED || j->state == HK_JOB_FAILED) {
            std::memset(rgb, 0, bytes);
            if (fraction) *fraction = 0.0;
            return HK_OK;
        }
        if (j->state == HK_JOB_DONE) {
            if (j->out) std::memcpy(rgb, j->out, bytes);
            if (fraction) *fraction = 1.0;
            return HK_OK;
        }
        j->preview_dst = rgb;
        j->preview_state = 1;
        s->cv_work.notify_all();
        // the job may also end meanwhile: then its final image is the preview
        auto ready = [&] { return j->preview_state == 2 || j->state >= HK_JOB_DONE; };
        bool ok = timeout_s < 0 ? (s->cv_done.wait(lk, ready), true)
                                : s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready);
        const bool written = j->preview_state == 2;
        j->preview_state = 0;
        j->preview_dst = nullptr;
        if (!ok) throw HkError{HK_ERR_TIMEOUT, "preview not ready within the timeout"};
        if (!written) {
            if (j->state == HK_JOB_DONE && j->out) std::memcpy(rgb, j->out, bytes);
            else std::memset(rgb, 0, bytes);
            if (fraction) *fraction = j->state == HK_JOB_DONE ? 1.0 : 0.0;
            return HK_OK;
        }
        if (fraction) *fraction = j->preview_fraction;
        return HK_OK;
    });
}

int hk_server_get_stats(hk_server *s, hk_server_stats *o) {
    return guarded([&] {
        if (!s || !o) throw HkError{HK_ERR_INVALID, "bad arguments"};
        std::lock_guard<std::mutex> lk(s->mu);
        std::memset(o, 0, sizeof *o);
        o->jobs_submitted = s->n_submitted;
        o->jobs_done = s->n_done;
        o->jobs_cancelled = s->n_cancelled;
        o->jobs_queued = s->n_queued;
        o->jobs_running = s->n_running;
        o->paths_done = s->paths_done;
        o->rays = s->rays;
        o->shadow_rays = s->shadow_rays;
        o->bytes_in_use = s->in_use;
        o->hbm_budget = s->budget;
        o->busy_s = s->busy_s;
        o->now_s = s->now();
        return HK_OK;
    });
}

}  // extern "C"
