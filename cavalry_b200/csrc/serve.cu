// Serving loop with continuous batching: render jobs and ray-query jobs of uneven size are
// admitted as they arrive (FIFO, under an HBM budget and a live-job limit), and every tick
// advances all live jobs by one bounce with ONE closest-hit and ONE any-hit traversal
// launch over the merged wavefronts of all of them (trace_*_segments: each segment is one
// job's rays against its own resident BVH).  Shading stays per job (its own kernels on the
// same stream).  Scenes and their BVHs are resident (cav_scene / cav_bvh handles owned by
// the caller); path state lives on the device for the job's lifetime.
//
// The reference renders one scene per process (main.cu:25-96) and has no request loop; the
// baseline for this component is the same loop with one live job at a time
// (CAV_SERVE_SEQUENTIAL), i.e. the plain sequential render loop over the same kernels.
//
// A dedicated host thread runs the loop; submissions and polls from other threads take a
// mutex.  Host buffers handed to a job must stay valid until the job is done.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cav_internal.cuh"

namespace {

using Clock = std::chrono::steady_clock;

enum JobKind { kRender = 0, kClosest = 1, kAny = 2 };

struct Job {
    int64_t id = 0;
    int kind = kRender;
    // render
    cav_scene* scene = nullptr;
    cav_render_opts opts{};
    float* host_sum = nullptr;
    float* host_weight = nullptr;
    cav::PathJob* pj = nullptr;
    // ray query
    const cav_bvh* bvh = nullptr;
    const cav_ray* h_rays = nullptr;
    const float* h_limit = nullptr;
    const int32_t* h_excl = nullptr;
    int64_t n = 0;
    int32_t* h_prim = nullptr;
    float* h_t = nullptr;
    float* h_uv = nullptr;
    uint8_t* h_occ = nullptr;
    void* dbuf = nullptr;
    cav_ray* d_rays = nullptr;
    float* d_limit = nullptr;
    int32_t* d_excl = nullptr;
    int32_t* d_prim = nullptr;
    float* d_t = nullptr;
    float* d_uv = nullptr;
    uint8_t* d_occ = nullptr;
    bool traced = false;
    // bookkeeping
    size_t bytes = 0;
    int state = CAV_JOB_PENDING;
    cav_status status = CAV_OK;
    double t_submit = 0, t_start = 0, t_done = 0;
    int64_t bounces = 0;
};

size_t ray_job_bytes(int kind, int64_t n) {
    size_t b = (size_t)n * sizeof(cav_ray) + 1024;
    if (kind == kClosest) b += (size_t)n * 16 + 512;
    else b += (size_t)n * 13 + 512;
    return b;
}

}  // namespace

struct cav_server {
    cav_ctx* ctx = nullptr;
    cav_server_config cfg{};
    cudaStream_t stream = nullptr;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv;       // work arrived / stop
    std::condition_variable done_cv;  // a job finished
    bool stop = false;
    std::deque<Job*> pending;
    std::vector<Job*> live;
    std::unordered_map<int64_t, Job*> jobs;
    int64_t next_id = 1;
    size_t used = 0;
    Clock::time_point t0;
    // segment tables: pinned host staging + device copies, one pair per traversal kind
    cav::TraceSeg* h_seg_c = nullptr;
    cav::TraceSeg* h_seg_a = nullptr;
    cav::TraceSeg* d_seg_c = nullptr;
    cav::TraceSeg* d_seg_a = nullptr;
    unsigned long long* d_counter = nullptr;  // traversal work counters (2)
    // statistics
    int64_t ticks = 0, closest_launches = 0, any_launches = 0, max_segments = 0;
    double busy_s = 0;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
    uint32_t trace_flags() const { return cfg.trace_flags & CAV_TRACE_FAST ? CAV_TRACE_FAST : CAV_TRACE_EXACT; }
    void run();
    void admit_locked(std::vector<Job*>& started);
    bool start(Job* j);
    void tick();
    void finish(Job* j, cav_status st);
};

void cav_server::admit_locked(std::vector<Job*>& started) {
    const int max_live = cfg.mode == CAV_SERVE_SEQUENTIAL ? 1 : (cfg.max_live_jobs > 0 ? cfg.max_live_jobs : 64);
    while (!pending.empty() && (int)live.size() + (int)started.size() < max_live) {
        Job* j = pending.front();
        const bool alone = live.empty() && started.empty();
        // FIFO under the HBM budget; a job larger than the whole budget runs alone
        if (!alone && used + j->bytes > (size_t)cfg.hbm_budget_bytes) break;
        pending.pop_front();
        used += j->bytes;
        j->state = CAV_JOB_RUNNING;
        started.push_back(j);
    }
}

bool cav_server::start(Job* j) {
    j->t_start = now();
    cav_status st = CAV_OK;
    const cav_bvh* tree = j->kind == kRender ? cav_scene_bvh(j->scene) : j->bvh;
    if (trace_flags() == CAV_TRACE_FAST) st = cav::ensure_wide(ctx, tree, stream);  // once per tree
    if (st != CAV_OK) {
        finish(j, st);
        return false;
    }
    if (j->kind == kRender) {
        st = cav::path_job_create(ctx, j->scene, &j->opts, stream, &j->pj);
    } else {
        if (cudaMallocAsync(&j->dbuf, j->bytes, stream) != cudaSuccess) {
            cudaGetLastError();
            st = CAV_ERR_OUT_OF_MEMORY;
        } else {
            unsigned char* p = (unsigned char*)j->dbuf;
            auto carve = [&](size_t b) {
                unsigned char* r = (unsigned char*)(((uintptr_t)p + 255) & ~(uintptr_t)255);
                p = r + b;
                return (void*)r;
            };
            j->d_rays = (cav_ray*)carve(sizeof(cav_ray) * j->n);
            cudaMemcpyAsync(j->d_rays, j->h_rays, sizeof(cav_ray) * j->n, cudaMemcpyHostToDevice, stream);
            if (j->kind == kClosest) {
                j->d_prim = (int32_t*)carve(4 * j->n);
                j->d_t = (float*)carve(4 * j->n);
                j->d_uv = (float*)carve(8 * j->n);
            } else {
                if (j->h_limit) {
                    j->d_limit = (float*)carve(4 * j->n);
                    cudaMemcpyAsync(j->d_limit, j->h_limit, 4 * j->n, cudaMemcpyHostToDevice, stream);
                }
                if (j->h_excl) {
                    j->d_excl = (int32_t*)carve(8 * j->n);
                    cudaMemcpyAsync(j->d_excl, j->h_excl, 8 * j->n, cudaMemcpyHostToDevice, stream);
                }
                j->d_occ = (uint8_t*)carve(j->n);
            }
        }
    }
    if (st != CAV_OK) {
        finish(j, st);
        return false;
    }
    return true;
}

void cav_server::finish(Job* j, cav_status st) {
    if (j->pj) {
        cav::path_job_destroy(j->pj, stream);
        j->pj = nullptr;
    }
    if (j->dbuf) {
        cudaFreeAsync(j->dbuf, stream);
        j->dbuf = nullptr;
    }
    std::lock_guard<std::mutex> lk(mu);
    used -= j->bytes;
    j->status = st;
    j->state = st == CAV_OK ? CAV_JOB_DONE : CAV_JOB_FAILED;
    j->t_done = now();
    done_cv.notify_all();
}

// One bounce of every live job: merged extend traversal, per-job shading, merged shadow
// traversal, per-job accumulation; finished jobs copy their results out.
void cav_server::tick() {
    const auto t_begin = Clock::now();
    ++ticks;
    cav_status err = CAV_OK;
    // ---- extend (closest hit): render jobs' current rays + closest-hit query jobs
    int nc = 0;
    int64_t total = 0;
    std::vector<Job*> in_c;
    for (Job* j : live) {
        cav::TraceSeg sg{};
        int64_t k = 0;
        if (j->kind == kRender) {
            k = cav::path_job_extend(j->pj, &sg);
        } else if (j->kind == kClosest && !j->traced) {
            const cav_bvh* b = j->bvh;
            sg.nodes = b->tnodes;
            sg.tris = b->tris;
            sg.cnodes = b->cnodes;
            sg.ctris = b->ctris;
            sg.root_box = b->d_root_box;
            sg.rays = j->d_rays;
            sg.prim = j->d_prim;
            sg.t = j->d_t;
            sg.uv = j->d_uv;
            k = j->n;
        }
        if (k <= 0) continue;
        if (nc == cav::trace_max_segments()) break;  // the rest waits for the next tick
        sg.begin = total;
        h_seg_c[nc++] = sg;
        total += k;
        in_c.push_back(j);
    }
    if (nc > 0) {
        max_segments = std::max<int64_t>(max_segments, nc);
        cudaMemcpyAsync(d_seg_c, h_seg_c, sizeof(cav::TraceSeg) * nc, cudaMemcpyHostToDevice, stream);
        err = cav::trace_closest_segments(ctx, d_seg_c, nc, total, trace_flags(), stream, d_counter);
        ++closest_launches;
    }
    std::vector<Job*> shaded;
    for (Job* j : in_c) {
        if (j->kind == kRender) {
            cav::path_job_shade(j->pj, stream);
            shaded.push_back(j);
        } else {
            j->traced = true;
        }
    }
    if (!shaded.empty()) cudaStreamSynchronize(stream);  // shadow-ray counts
    // ---- shadow (any hit): render jobs' shadow rays + any-hit query jobs
    int na = 0;
    total = 0;
    std::vector<Job*> in_a;
    for (Job* j : live) {
        cav::TraceSeg sg{};
        int64_t k = 0;
        if (j->kind == kRender) {
            if (std::find(shaded.begin(), shaded.end(), j) == shaded.end()) continue;
            k = cav::path_job_shadow(j->pj, &sg);
        } else if (j->kind == kAny && !j->traced) {
            const cav_bvh* b = j->bvh;
            sg.nodes = b->tnodes;
            sg.tris = b->tris;
            sg.cnodes = b->cnodes;
            sg.ctris = b->ctris;
            sg.root_box = b->d_root_box;
            sg.rays = j->d_rays;
            sg.limit = j->d_limit;
            sg.excl = j->d_excl;
            sg.occ = j->d_occ;
            k = j->n;
        }
        if (k <= 0) continue;
        if (na == cav::trace_max_segments()) break;
        sg.begin = total;
        h_seg_a[na++] = sg;
        total += k;
        in_a.push_back(j);
    }
    if (na > 0 && err == CAV_OK) {
        cudaMemcpyAsync(d_seg_a, h_seg_a, sizeof(cav::TraceSeg) * na, cudaMemcpyHostToDevice, stream);
        err = cav::trace_any_segments(ctx, d_seg_a, na, total, trace_flags(), stream, d_counter + 1);
        ++any_launches;
    }
    for (Job* j : in_a)
        if (j->kind == kAny) j->traced = true;
    // ---- advance render jobs; results of finished jobs
    std::vector<Job*> done;
    for (Job* j : shaded) {
        bool fin = false;
        cav::path_job_advance(j->pj, stream, &fin);
        ++j->bounces;
        if (fin) {
            float *s, *w;
            int64_t px;
            cav::path_job_film(j->pj, &s, &w, &px);
            cudaMemcpyAsync(j->host_sum, s, sizeof(float) * 3 * px, cudaMemcpyDeviceToHost, stream);
            cudaMemcpyAsync(j->host_weight, w, sizeof(float) * px, cudaMemcpyDeviceToHost, stream);
            done.push_back(j);
        }
    }
    for (Job* j : live) {
        if (j->kind == kRender || !j->traced) continue;
        if (j->kind == kClosest) {
            cudaMemcpyAsync(j->h_prim, j->d_prim, 4 * j->n, cudaMemcpyDeviceToHost, stream);
            if (j->h_t) cudaMemcpyAsync(j->h_t, j->d_t, 4 * j->n, cudaMemcpyDeviceToHost, stream);
            if (j->h_uv) cudaMemcpyAsync(j->h_uv, j->d_uv, 8 * j->n, cudaMemcpyDeviceToHost, stream);
        } else {
            cudaMemcpyAsync(j->h_occ, j->d_occ, j->n, cudaMemcpyDeviceToHost, stream);
        }
        done.push_back(j);
    }
    cudaError_t ce = cudaStreamSynchronize(stream);
    if (ce != cudaSuccess && err == CAV_OK) err = cav::cuda_error(ctx, ce, "serve tick");
    if (err != CAV_OK) {  // a failed launch fails every live job
        std::vector<Job*> all;
        {
            std::lock_guard<std::mutex> lk(mu);
            all.swap(live);
        }
        for (Job* j : all) finish(j, err);
        return;
    }
    for (Job* j : done) {
        {
            std::lock_guard<std::mutex> lk(mu);
            live.erase(std::find(live.begin(), live.end(), j));
        }
        finish(j, CAV_OK);
    }
    busy_s += std::chrono::duration<double>(Clock::now() - t_begin).count();
}

void cav_server::run() {
    cudaSetDevice(ctx->device);
    for (;;) {
        std::vector<Job*> started;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return stop || !pending.empty() || !live.empty(); });
            if (stop && live.empty()) {
                for (Job* j : pending) {  // never started
                    j->state = CAV_JOB_FAILED;
                    j->status = CAV_ERR_NOT_READY;
                    j->t_done = now();
                }
                pending.clear();
                done_cv.notify_all();
                return;
            }
            if (!stop) admit_locked(started);
        }
        for (Job* j : started)
            if (start(j)) {
                std::lock_guard<std::mutex> lk(mu);
                live.push_back(j);
            }
        if (!live.empty()) tick();
    }
}

// ================================================================================ C ABI
extern "C" {

cav_status cav_server_create(cav_ctx* ctx, const cav_server_config* cfg, cav_server** out) {
    if (!ctx || !out) return CAV_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return cav::cuda_error(ctx, cudaGetLastError(), "cudaSetDevice");
    auto* sv = new cav_server();
    sv->ctx = ctx;
    sv->cfg.hbm_budget_bytes = (int64_t)80 << 30;
    sv->cfg.mode = CAV_SERVE_MERGED;
    sv->cfg.max_live_jobs = 64;
    sv->cfg.max_paths_per_job = (int64_t)1 << 20;
    if (cfg) {
        if (cfg->hbm_budget_bytes > 0) sv->cfg.hbm_budget_bytes = cfg->hbm_budget_bytes;
        sv->cfg.mode = cfg->mode;
        if (cfg->max_live_jobs > 0) sv->cfg.max_live_jobs = cfg->max_live_jobs;
        if (cfg->max_paths_per_job > 0) sv->cfg.max_paths_per_job = cfg->max_paths_per_job;
        sv->cfg.trace_flags = cfg->trace_flags;
    }
    const int ms = cav::trace_max_segments();
    cudaError_t e = cudaStreamCreateWithFlags(&sv->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost(&sv->h_seg_c, sizeof(cav::TraceSeg) * ms);
    if (e == cudaSuccess) e = cudaMallocHost(&sv->h_seg_a, sizeof(cav::TraceSeg) * ms);
    if (e == cudaSuccess) e = cudaMalloc(&sv->d_seg_c, sizeof(cav::TraceSeg) * ms);
    if (e == cudaSuccess) e = cudaMalloc(&sv->d_seg_a, sizeof(cav::TraceSeg) * ms);
    if (e == cudaSuccess) e = cudaMalloc(&sv->d_counter, 64);
    if (e != cudaSuccess) {
        cav_server_destroy(sv);
        return cav::cuda_error(ctx, e, "cav_server_create");
    }
    sv->t0 = Clock::now();
    sv->worker = std::thread([sv] { sv->run(); });
    *out = sv;
    return CAV_OK;
}

cav_status cav_server_destroy(cav_server* sv) {
    if (!sv) return CAV_OK;
    if (sv->worker.joinable()) {
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            sv->stop = true;
        }
        sv->cv.notify_all();
        sv->worker.join();
    }
    if (sv->stream) cudaStreamSynchronize(sv->stream);
    for (auto& kv : sv->jobs) delete kv.second;
    cudaFreeHost(sv->h_seg_c);
    cudaFreeHost(sv->h_seg_a);
    cudaFree(sv->d_seg_c);
    cudaFree(sv->d_seg_a);
    cudaFree(sv->d_counter);
    if (sv->stream) cudaStreamDestroy(sv->stream);
    delete sv;
    return CAV_OK;
}

static cav_status enqueue(cav_server* sv, Job* j, int64_t* id) {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) {
        delete j;
        return CAV_ERR_NOT_READY;
    }
    j->id = sv->next_id++;
    j->t_submit = sv->now();
    sv->jobs[j->id] = j;
    sv->pending.push_back(j);
    *id = j->id;
    sv->cv.notify_all();
    return CAV_OK;
}

cav_status cav_server_submit_render(cav_server* sv, cav_scene* scene, const cav_render_opts* opts, float* host_sum,
                                    float* host_weight, int64_t* job_id) {
    if (!sv || !scene || !host_sum || !host_weight || !job_id) return CAV_ERR_INVALID_ARGUMENT;
    cav_scene_info_t info;
    cav_scene_info(scene, &info);
    const int integrator = opts && opts->integrator != 0 ? opts->integrator : info.integrator;
    if (integrator == 1) return cav::set_error(sv->ctx, CAV_ERR_INVALID_ARGUMENT, "the server renders the path integrator");
    auto* j = new Job();
    j->kind = kRender;
    j->scene = scene;
    if (opts) j->opts = *opts;
    j->host_sum = host_sum;
    j->host_weight = host_weight;
    if (j->opts.max_paths_in_flight <= 0) j->opts.max_paths_in_flight = sv->cfg.max_paths_per_job;
    j->bytes = cav::path_job_bytes(scene, &j->opts);
    return enqueue(sv, j, job_id);
}

cav_status cav_server_submit_rays(cav_server* sv, const cav_bvh* bvh, int any_hit, const cav_ray* host_rays,
                                  const float* host_limit, const int32_t* host_excl, int64_t n, int32_t* host_prim,
                                  float* host_t, float* host_uv, uint8_t* host_occ, int64_t* job_id) {
    if (!sv || !bvh || !host_rays || n <= 0 || !job_id) return CAV_ERR_INVALID_ARGUMENT;
    if (any_hit ? !host_occ : !host_prim) return CAV_ERR_INVALID_ARGUMENT;
    auto* j = new Job();
    j->kind = any_hit ? kAny : kClosest;
    j->bvh = bvh;
    j->h_rays = host_rays;
    j->h_limit = host_limit;
    j->h_excl = host_excl;
    j->n = n;
    j->h_prim = host_prim;
    j->h_t = host_t;
    j->h_uv = host_uv;
    j->h_occ = host_occ;
    j->bytes = ray_job_bytes(j->kind, n);
    return enqueue(sv, j, job_id);
}

static void fill_status(const Job* j, cav_job_status* st) {
    st->state = j->state;
    st->status = j->status;
    st->t_submit = j->t_submit;
    st->t_start = j->t_start;
    st->t_done = j->t_done;
    st->bounces = j->bounces;
}

cav_status cav_server_poll(cav_server* sv, int64_t job_id, cav_job_status* st) {
    if (!sv || !st) return CAV_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(job_id);
    if (it == sv->jobs.end()) return CAV_ERR_INVALID_ARGUMENT;
    fill_status(it->second, st);
    return CAV_OK;
}

cav_status cav_server_wait(cav_server* sv, int64_t job_id, double timeout_s, cav_job_status* st) {
    if (!sv) return CAV_ERR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(job_id);
    if (it == sv->jobs.end()) return CAV_ERR_INVALID_ARGUMENT;
    Job* j = it->second;
    auto pred = [&] { return j->state == CAV_JOB_DONE || j->state == CAV_JOB_FAILED; };
    if (timeout_s < 0) sv->done_cv.wait(lk, pred);
    else if (!sv->done_cv.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) return CAV_ERR_TIMEOUT;
    if (st) fill_status(j, st);
    return j->status;
}

cav_status cav_server_stats(cav_server* sv, cav_server_stats_t* out) {
    if (!sv || !out) return CAV_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(sv->mu);
    out->ticks = sv->ticks;
    out->closest_launches = sv->closest_launches;
    out->any_launches = sv->any_launches;
    out->max_segments = sv->max_segments;
    out->busy_s = sv->busy_s;
    out->now_s = sv->now();
    out->pending = (int64_t)sv->pending.size();
    out->live = (int64_t)sv->live.size();
    out->hbm_in_use = (int64_t)sv->used;
    return CAV_OK;
}

}  // extern "C"
