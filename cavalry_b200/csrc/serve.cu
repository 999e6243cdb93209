// Serving loop with continuous batching: render jobs and ray-query jobs of uneven size are
// admitted as they arrive (FIFO, under an HBM budget and a live-job limit), and every tick
// advances all live jobs of a lane by one bounce with ONE closest-hit and ONE any-hit
// traversal launch over the merged wavefronts of all of them (trace_*_segments: each
// segment is one job's rays against its own BVH).  Shading stays per job (its own kernels
// on the lane's stream); path state lives on the device for the job's lifetime.
//
// Scenes: a job either names a resident scene or tree (cav_scene / cav_bvh handles owned
// by the caller) or brings its own .pbrt file (cav_server_submit_scene).  Loader threads
// parse those files as they arrive; the lane that admits such a job uploads its scene
// stream-ordered, builds the trees of all scenes it admitted in that round with one
// batched build (per treelet round count), and releases the scene when the job ends.
// Small renders (at most graph_max_paths paths) are replayed as one CUDA graph of the whole
// render instead of joining the per-tick merged launches.  Jobs can be cancelled (pending:
// dropped; running: removed by their lane before its next bounce), and a job whose
// estimated bytes exceed the HBM budget can be refused at submission.
//
// Lanes: a few host threads, each with its own stream and share of the live jobs, tick
// independently, so the GPU runs one lane's traversal while the other lane's launches
// drain their tails, its per-job kernels run and its host waits for queue counts.
//
// The reference renders one scene per process (main.cu:25-96) and has no request loop; the
// baseline for this component is the plain sequential loop of cav_render calls (and
// CAV_SERVE_SEQUENTIAL, one live job at a time, the same loop inside the server).
//
// Submissions and polls from other threads take a mutex.  Host buffers handed to a job
// must stay valid until the job is done.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cav_internal.cuh"
#include "pbrt.h"

namespace {

using Clock = std::chrono::steady_clock;

enum JobKind { kRender = 0, kClosest = 1, kAny = 2 };

struct Job {
    int64_t id = 0;
    int kind = kRender;
    // a scene the job brings (cav_server_submit_scene): parsed by a loader thread, uploaded
    // and built by the lane that admits the job, released when the job ends
    bool owns_scene = false;
    std::string path;
    int rounds = -1;
    std::unique_ptr<cavpbrt::Scene> desc;
    bool graph = false;            // render replayed as one CUDA graph instead of per-tick bounces
    bool graph_launched = false;
    float* d_film = nullptr;       // the graph render's device film
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
    std::atomic<bool> cancel{false};  // set by cav_server_cancel while the job runs
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

// One lane: a host thread with its own stream, live jobs and segment tables.  Lanes tick
// independently and share the GPU, so one lane's launch tails and small per-job kernels
// overlap the other lane's traversal.
struct Lane {
    int index = 0;
    cudaStream_t stream = nullptr;
    std::thread worker;
    std::vector<Job*> live;  // changed by the lane's own thread, under the server mutex
    // segment tables: pinned host staging + device copies, one pair per traversal kind
    cav::TraceSeg* h_seg_c = nullptr;
    cav::TraceSeg* h_seg_a = nullptr;
    cav::TraceSeg* d_seg_c = nullptr;
    cav::TraceSeg* d_seg_a = nullptr;
    unsigned long long* d_counter = nullptr;  // traversal work counters (2)
};

struct cav_server {
    cav_ctx* ctx = nullptr;
    cav_server_config cfg{};
    std::vector<Lane*> lanes;
    std::mutex mu;
    std::condition_variable cv;       // work arrived / memory freed / stop
    std::condition_variable done_cv;  // a job finished
    bool stop = false;
    std::deque<Job*> pending;
    std::deque<Job*> to_parse;          // scene jobs waiting for a loader thread
    std::vector<std::thread> loaders;   // host threads parsing the scenes jobs bring
    std::condition_variable loader_cv;
    std::unordered_map<int64_t, Job*> jobs;
    int64_t next_id = 1;
    size_t used = 0;
    Clock::time_point t0;
    // statistics (under mu)
    int64_t ticks = 0, closest_launches = 0, any_launches = 0, max_segments = 0;
    double busy_s = 0;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
    uint32_t trace_flags() const { return cfg.trace_flags & CAV_TRACE_FAST ? CAV_TRACE_FAST : CAV_TRACE_EXACT; }
    int lane_limit() const {  // live jobs a lane keeps
        if (cfg.mode == CAV_SERVE_SEQUENTIAL) return 1;
        const int total = cfg.max_live_jobs > 0 ? cfg.max_live_jobs : 64;
        const int nl = (int)lanes.size();
        return std::max(1, (total + nl - 1) / nl);
    }
    int64_t live_count_locked() const {
        int64_t k = 0;
        for (const Lane* l : lanes) k += (int64_t)l->live.size();
        return k;
    }
    int live_renders_locked() const {
        int k = 0;
        for (const Lane* l : lanes)
            for (const Job* j : l->live) k += j->kind == kRender;
        return k;
    }
    // Paths a render job's next chunk starts: the live render jobs share one job's capacity,
    // but no slice drops below the configured floor (or the capacity, when that is smaller).
    // A job alone runs chunks as large as cav_render's; many jobs advance in shorter ticks.
    int64_t slice_for(int64_t capacity, int renders) const {
        const int64_t floor_paths = std::min<int64_t>(capacity, cfg.min_paths_per_slice);
        return std::max(floor_paths, capacity / std::max(renders, 1));
    }
    bool can_admit_locked(const Lane* l) const;
    void run(Lane* l);
    void load();
    void admit_locked(Lane* l, std::vector<Job*>& started);
    bool upload(Lane* l, Job* j);
    void build_trees(Lane* l, std::vector<Job*>& jobs);
    bool start(Lane* l, Job* j);
    void tick(Lane* l);
    void finish(Lane* l, Job* j, cav_status st);
};

bool cav_server::can_admit_locked(const Lane* l) const {
    if (pending.empty() || (int)l->live.size() >= lane_limit()) return false;
    // FIFO under the HBM budget; a job larger than the whole budget runs alone
    return live_count_locked() == 0 || used + pending.front()->bytes <= (size_t)cfg.hbm_budget_bytes;
}

void cav_server::admit_locked(Lane* l, std::vector<Job*>& started) {
    const int limit = lane_limit();
    while (!pending.empty() && (int)l->live.size() + (int)started.size() < limit) {
        Job* j = pending.front();
        const bool alone = live_count_locked() == 0 && started.empty();
        if (!alone && used + j->bytes > (size_t)cfg.hbm_budget_bytes) break;
        pending.pop_front();
        used += j->bytes;
        j->state = CAV_JOB_RUNNING;
        started.push_back(j);
    }
}

// Loader thread: parses the scenes that jobs bring (host work that overlaps the device work
// of the jobs already running), sizes each job's device memory and queues it for admission.
void cav_server::load() {
    for (;;) {
        Job* j = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu);
            loader_cv.wait(lk, [&] { return stop || !to_parse.empty(); });
            if (stop) return;  // cav_server_destroy fails what is still queued
            j = to_parse.front();
            to_parse.pop_front();
        }
        auto d = std::make_unique<cavpbrt::Scene>();
        cav_status st = CAV_OK;
        try {
            *d = cavpbrt::load_file(j->path, cavpbrt::Overrides{});
        } catch (const std::exception&) {
            st = CAV_ERR_INVALID_ARGUMENT;
        }
        size_t bytes = 0;
        if (st == CAV_OK) {
            bytes = cav::scene_device_bytes(*d);
            if (j->kind == kRender) {
                const int spp = j->opts.spp > 0 ? j->opts.spp : d->spp;
                const int64_t total = (int64_t)j->opts.width * j->opts.height * spp;
                j->graph = cfg.graph_max_paths > 0 && total <= cfg.graph_max_paths;
                bytes += cav::render_state_bytes(j->opts.width, j->opts.height, spp,
                                                 j->graph ? 0 : j->opts.max_paths_in_flight);
            } else {
                bytes += ray_job_bytes(j->kind, j->n);
            }
            if (cfg.reject_over_budget && bytes > (size_t)cfg.hbm_budget_bytes) st = CAV_ERR_OUT_OF_MEMORY;
        }
        std::lock_guard<std::mutex> lk(mu);
        if (j->state == CAV_JOB_CANCELLED) continue;  // cancelled while it was parsed
        if (st != CAV_OK) {
            j->state = CAV_JOB_FAILED;
            j->status = st;
            j->t_done = now();
            done_cv.notify_all();
            continue;
        }
        j->desc = std::move(d);
        j->bytes = bytes;
        pending.push_back(j);
        cv.notify_all();
    }
}

// A scene job's scene: uploaded on the lane's stream (stream-ordered allocations and copies).
bool cav_server::upload(Lane* l, Job* j) {
    j->t_start = now();
    cav_scene* sc = nullptr;
    cav_status st = cav::scene_upload(ctx, std::move(*j->desc), l->stream, true, &sc);
    j->desc.reset();
    if (st != CAV_OK) {
        finish(l, j, st);
        return false;
    }
    j->scene = sc;
    if (j->rounds < 0) {  // the reference's default (Core/Scene.cu:141-146)
        const int spp = j->kind == kRender && j->opts.spp > 0 ? j->opts.spp : cav::scene_spp(sc);
        j->rounds = spp >= 64 ? 10 : 3;
    }
    return true;
}

// The trees of the scenes admitted together: one batched build (one launch per LBVH stage
// over all of them) per treelet-round count.  Jobs whose build fails are finished here.
void cav_server::build_trees(Lane* l, std::vector<Job*>& js) {
    std::vector<Job*> ok;
    std::vector<int> rounds_seen;
    for (Job* j : js)
        if (std::find(rounds_seen.begin(), rounds_seen.end(), j->rounds) == rounds_seen.end())
            rounds_seen.push_back(j->rounds);
    for (int rounds : rounds_seen) {
        std::vector<Job*> g;
        for (Job* j : js)
            if (j->rounds == rounds) g.push_back(j);
        const int K = (int)g.size();
        std::vector<const float*> pos(K);
        std::vector<const int32_t*> idx(K), mesh(K);
        std::vector<int64_t> nv(K), nt(K);
        std::vector<cav_bvh*> out(K, nullptr);
        for (int k = 0; k < K; ++k) cav::scene_geometry(g[k]->scene, &pos[k], &nv[k], &idx[k], &mesh[k], &nt[k]);
        const cav_status st =
            K == 1 ? cav::build_bvh(ctx, pos[0], nv[0], idx[0], mesh[0], nt[0], nullptr, rounds, l->stream, &out[0])
                   : cav::build_bvh_batch(ctx, K, pos.data(), nv.data(), idx.data(), mesh.data(), nt.data(), nullptr,
                                          rounds, l->stream, out.data());
        for (int k = 0; k < K; ++k) {
            if (st == CAV_OK) {
                cav::scene_set_bvh(g[k]->scene, out[k], rounds);
                ok.push_back(g[k]);
            } else {
                finish(l, g[k], st);
            }
        }
    }
    js.swap(ok);
}

bool cav_server::start(Lane* l, Job* j) {
    if (!j->owns_scene) j->t_start = now();
    cav_status st = CAV_OK;
    const cudaStream_t stream = l->stream;
    if (j->owns_scene && j->kind != kRender) j->bvh = cav_scene_bvh(j->scene);
    const cav_bvh* tree = j->kind == kRender ? cav_scene_bvh(j->scene) : j->bvh;
    if (trace_flags() == CAV_TRACE_FAST) st = cav::ensure_wide(ctx, tree, stream);  // once per tree
    if (st != CAV_OK) {
        finish(l, j, st);
        return false;
    }
    if (j->graph) {
        // a small render: its whole bounce chain replayed as one CUDA graph on the lane's
        // stream (no per-bounce host round trip); the copies to pageable host memory return
        // once the film is on the host, so the job ends here
        const int64_t px = (int64_t)j->opts.width * j->opts.height;
        cav_render_opts o = j->opts;
        if (trace_flags() == CAV_TRACE_FAST) o.flags |= CAV_RENDER_FAST_TRACE;
        if (cav::dev_alloc(ctx, (void**)&j->d_film, sizeof(float) * 4 * px, stream, true) != cudaSuccess) {
            cudaGetLastError();
            finish(l, j, CAV_ERR_OUT_OF_MEMORY);
            return false;
        }
        cudaMemsetAsync(j->d_film, 0, sizeof(float) * 4 * px, stream);
        st = cav::render_path_graph(ctx, j->scene, &o, j->d_film, j->d_film + 3 * px, stream, l->d_counter + 2);
        if (st == CAV_OK) {
            cudaError_t e = cudaMemcpyAsync(j->host_sum, j->d_film, sizeof(float) * 3 * px, cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(j->host_weight, j->d_film + 3 * px, sizeof(float) * px, cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) st = cav::cuda_error(ctx, e, "graph render job");
        }
        ++j->bounces;
        finish(l, j, st);
        return false;
    }
    if (j->kind == kRender) {
        int renders;
        {
            std::lock_guard<std::mutex> lk(mu);
            renders = 1 + live_renders_locked();
        }
        st = cav::path_job_create(ctx, j->scene, &j->opts, slice_for(j->opts.max_paths_in_flight, renders), stream,
                                  &j->pj);
    } else {
        if (cav::dev_alloc(ctx, &j->dbuf, j->bytes, stream, true) != cudaSuccess) {
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
        finish(l, j, st);
        return false;
    }
    return true;
}

void cav_server::finish(Lane* l, Job* j, cav_status st) {
    if (j->pj) {
        cav::path_job_destroy(j->pj, l->stream);
        j->pj = nullptr;
    }
    if (j->dbuf) {
        cudaFreeAsync(j->dbuf, l->stream);
        j->dbuf = nullptr;
    }
    if (j->d_film) {
        cudaFreeAsync(j->d_film, l->stream);
        j->d_film = nullptr;
    }
    if (j->owns_scene && j->scene) {  // the scene (and its tree) the job brought
        cav::scene_release(j->scene, l->stream, true);
        j->scene = nullptr;
        j->bvh = nullptr;
    }
    j->desc.reset();
    std::lock_guard<std::mutex> lk(mu);
    used -= j->bytes;
    j->status = st;
    j->state = st == CAV_OK ? CAV_JOB_DONE : st == CAV_ERR_CANCELLED ? CAV_JOB_CANCELLED : CAV_JOB_FAILED;
    j->t_done = now();
    done_cv.notify_all();
    cv.notify_all();  // memory came free: another lane may admit
}

// One bounce of every live job of the lane: merged extend traversal, per-job shading,
// merged shadow traversal, per-job accumulation; finished jobs copy their results out.
void cav_server::tick(Lane* l) {
    const auto t_begin = Clock::now();
    const cudaStream_t stream = l->stream;
    std::vector<Job*>& live = l->live;
    // cancelled jobs leave before the tick: their last work on this stream has completed
    // (every tick ends with a stream synchronisation), so their state is freed in order
    std::vector<Job*> cancelled;
    {
        std::lock_guard<std::mutex> lk(mu);
        for (Job* j : live)
            if (j->cancel.load()) cancelled.push_back(j);
        for (Job* j : cancelled) live.erase(std::find(live.begin(), live.end(), j));
    }
    for (Job* j : cancelled) finish(l, j, CAV_ERR_CANCELLED);
    if (live.empty()) return;
    cav_status err = CAV_OK;
    int64_t segs_c = 0, launches_c = 0, launches_a = 0;
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
        l->h_seg_c[nc++] = sg;
        total += k;
        in_c.push_back(j);
    }
    if (nc > 0) {
        segs_c = nc;
        cudaMemcpyAsync(l->d_seg_c, l->h_seg_c, sizeof(cav::TraceSeg) * nc, cudaMemcpyHostToDevice, stream);
        err = cav::trace_closest_segments(ctx, l->d_seg_c, nc, total, trace_flags(), stream, l->d_counter);
        ++launches_c;
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
        l->h_seg_a[na++] = sg;
        total += k;
        in_a.push_back(j);
    }
    if (na > 0 && err == CAV_OK) {
        cudaMemcpyAsync(l->d_seg_a, l->h_seg_a, sizeof(cav::TraceSeg) * na, cudaMemcpyHostToDevice, stream);
        err = cav::trace_any_segments(ctx, l->d_seg_a, na, total, trace_flags(), stream, l->d_counter + 1);
        ++launches_a;
    }
    for (Job* j : in_a)
        if (j->kind == kAny) j->traced = true;
    // ---- advance render jobs; results of finished jobs
    std::vector<Job*> done;
    int renders;
    {
        std::lock_guard<std::mutex> lk(mu);
        renders = live_renders_locked();
    }
    for (Job* j : shaded) {
        bool fin = false;
        cav::path_job_set_slice(j->pj, slice_for(cav::path_job_capacity(j->pj), renders));
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
    {
        std::lock_guard<std::mutex> lk(mu);
        ++ticks;
        closest_launches += launches_c;
        any_launches += launches_a;
        max_segments = std::max(max_segments, segs_c);
    }
    if (err != CAV_OK) {  // a failed launch fails every live job of the lane
        std::vector<Job*> all;
        {
            std::lock_guard<std::mutex> lk(mu);
            all.swap(live);
        }
        for (Job* j : all) finish(l, j, err);
        return;
    }
    for (Job* j : done) {
        {
            std::lock_guard<std::mutex> lk(mu);
            live.erase(std::find(live.begin(), live.end(), j));
        }
        finish(l, j, CAV_OK);
    }
    const double dt = std::chrono::duration<double>(Clock::now() - t_begin).count();
    std::lock_guard<std::mutex> lk(mu);
    busy_s += dt;
}

void cav_server::run(Lane* l) {
    cudaSetDevice(ctx->device);
    for (;;) {
        std::vector<Job*> started;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return stop || !l->live.empty() || can_admit_locked(l); });
            if (stop && l->live.empty()) {
                for (Job* j : pending) {  // never started
                    j->state = CAV_JOB_FAILED;
                    j->status = CAV_ERR_NOT_READY;
                    j->t_done = now();
                }
                pending.clear();
                done_cv.notify_all();
                return;
            }
            if (!stop) admit_locked(l, started);
        }
        // jobs that bring a scene: upload each, then build all their trees together
        std::vector<Job*> owned, ready;
        for (Job* j : started) {
            if (!j->owns_scene) ready.push_back(j);
            else if (upload(l, j)) owned.push_back(j);
        }
        if (!owned.empty()) build_trees(l, owned);
        ready.insert(ready.end(), owned.begin(), owned.end());
        for (Job* j : ready)
            if (start(l, j)) {
                std::lock_guard<std::mutex> lk(mu);
                l->live.push_back(j);
            }
        if (!l->live.empty()) tick(l);
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
    sv->cfg.max_paths_per_job = (int64_t)1 << 22;
    if (cfg) {
        if (cfg->hbm_budget_bytes > 0) sv->cfg.hbm_budget_bytes = cfg->hbm_budget_bytes;
        sv->cfg.mode = cfg->mode;
        if (cfg->max_live_jobs > 0) sv->cfg.max_live_jobs = cfg->max_live_jobs;
        if (cfg->max_paths_per_job > 0) sv->cfg.max_paths_per_job = cfg->max_paths_per_job;
        sv->cfg.trace_flags = cfg->trace_flags;
        sv->cfg.reject_over_budget = cfg->reject_over_budget;
    }
    sv->cfg.loaders = cfg && cfg->loaders > 0 ? std::min(cfg->loaders, 64) : 4;
    sv->cfg.graph_max_paths = !cfg || cfg->graph_max_paths == 0 ? (int64_t)1 << 18
                              : cfg->graph_max_paths < 0   ? 0
                                                           : cfg->graph_max_paths;
    sv->cfg.min_paths_per_slice = cfg && cfg->min_paths_per_slice > 0 ? cfg->min_paths_per_slice : (int64_t)1 << 22;
    int nl = cfg && cfg->lanes > 0 ? std::min(cfg->lanes, 8) : 1;
    if (sv->cfg.mode == CAV_SERVE_SEQUENTIAL) nl = 1;
    sv->cfg.lanes = nl;
    const int ms = cav::trace_max_segments();
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < nl && e == cudaSuccess; ++k) {
        auto* l = new Lane();
        l->index = k;
        sv->lanes.push_back(l);
        e = cudaStreamCreateWithFlags(&l->stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaMallocHost(&l->h_seg_c, sizeof(cav::TraceSeg) * ms);
        if (e == cudaSuccess) e = cudaMallocHost(&l->h_seg_a, sizeof(cav::TraceSeg) * ms);
        if (e == cudaSuccess) e = cudaMalloc(&l->d_seg_c, sizeof(cav::TraceSeg) * ms);
        if (e == cudaSuccess) e = cudaMalloc(&l->d_seg_a, sizeof(cav::TraceSeg) * ms);
        if (e == cudaSuccess) e = cudaMalloc(&l->d_counter, 64);
    }
    if (e != cudaSuccess) {
        cav_server_destroy(sv);
        return cav::cuda_error(ctx, e, "cav_server_create");
    }
    sv->t0 = Clock::now();
    for (Lane* l : sv->lanes) l->worker = std::thread([sv, l] { sv->run(l); });
    for (int k = 0; k < sv->cfg.loaders; ++k) sv->loaders.emplace_back([sv] { sv->load(); });
    *out = sv;
    return CAV_OK;
}

cav_status cav_server_destroy(cav_server* sv) {
    if (!sv) return CAV_OK;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->cv.notify_all();
    sv->loader_cv.notify_all();
    for (Lane* l : sv->lanes)
        if (l->worker.joinable()) l->worker.join();
    for (std::thread& t : sv->loaders)
        if (t.joinable()) t.join();
    {  // jobs still being parsed or queued when the server stopped never ran
        std::lock_guard<std::mutex> lk(sv->mu);
        for (auto& kv : sv->jobs) {
            Job* j = kv.second;
            if (j->state == CAV_JOB_PENDING) {
                j->state = CAV_JOB_FAILED;
                j->status = CAV_ERR_NOT_READY;
                j->t_done = sv->now();
            }
        }
        sv->done_cv.notify_all();
    }
    for (Lane* l : sv->lanes)
        if (l->stream) cudaStreamSynchronize(l->stream);
    for (auto& kv : sv->jobs) delete kv.second;
    for (Lane* l : sv->lanes) {
        cudaFreeHost(l->h_seg_c);
        cudaFreeHost(l->h_seg_a);
        cudaFree(l->d_seg_c);
        cudaFree(l->d_seg_a);
        cudaFree(l->d_counter);
        if (l->stream) cudaStreamDestroy(l->stream);
        delete l;
    }
    delete sv;
    return CAV_OK;
}

static cav_status enqueue(cav_server* sv, Job* j, int64_t* id) {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) {
        delete j;
        return CAV_ERR_NOT_READY;
    }
    if (sv->cfg.reject_over_budget && j->bytes > (size_t)sv->cfg.hbm_budget_bytes) {
        const size_t need = j->bytes;
        delete j;
        return cav::set_error(sv->ctx, CAV_ERR_OUT_OF_MEMORY,
                              "job rejected: it needs " + std::to_string(need) + " bytes of device memory, more than "
                              "the server's whole HBM budget");
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

cav_status cav_server_submit_scene(cav_server* sv, const cav_scene_job* spec, int64_t* job_id) {
    if (!sv || !spec || !spec->pbrt_path || !job_id) return CAV_ERR_INVALID_ARGUMENT;
    auto* j = new Job();
    j->owns_scene = true;
    j->path = spec->pbrt_path;
    j->rounds = spec->bvh_rounds;
    if (spec->kind == CAV_SCENE_RENDER) {
        if (!spec->host_sum || !spec->host_weight || spec->render.width <= 0 || spec->render.height <= 0 ||
            spec->render.integrator > 0) {
            delete j;
            return cav::set_error(sv->ctx, CAV_ERR_INVALID_ARGUMENT,
                                  "scene render job: films, width and height are required (path integrator)");
        }
        j->kind = kRender;
        j->opts = spec->render;
        j->host_sum = spec->host_sum;
        j->host_weight = spec->host_weight;
        if (j->opts.max_paths_in_flight <= 0) j->opts.max_paths_in_flight = sv->cfg.max_paths_per_job;
    } else if (spec->kind == CAV_SCENE_CLOSEST || spec->kind == CAV_SCENE_ANY) {
        const bool any = spec->kind == CAV_SCENE_ANY;
        if (!spec->host_rays || spec->n_rays <= 0 || (any ? !spec->host_occ : !spec->host_prim)) {
            delete j;
            return cav::set_error(sv->ctx, CAV_ERR_INVALID_ARGUMENT, "scene ray job: rays and outputs are required");
        }
        j->kind = any ? kAny : kClosest;
        j->h_rays = spec->host_rays;
        j->h_limit = spec->host_limit;
        j->h_excl = spec->host_excl;
        j->n = spec->n_rays;
        j->h_prim = spec->host_prim;
        j->h_t = spec->host_t;
        j->h_uv = spec->host_uv;
        j->h_occ = spec->host_occ;
    } else {
        delete j;
        return cav::set_error(sv->ctx, CAV_ERR_INVALID_ARGUMENT, "scene job: unknown kind");
    }
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) {
        delete j;
        return CAV_ERR_NOT_READY;
    }
    j->id = sv->next_id++;
    j->t_submit = sv->now();
    sv->jobs[j->id] = j;
    sv->to_parse.push_back(j);
    *job_id = j->id;
    sv->loader_cv.notify_one();
    return CAV_OK;
}

static void fill_status(const Job* j, cav_job_status* st) {
    st->state = j->state;
    st->status = j->status;
    st->t_submit = j->t_submit;
    st->t_start = j->t_start;
    st->t_done = j->t_done;
    st->bounces = j->bounces;
}

cav_status cav_server_cancel(cav_server* sv, int64_t job_id) {
    if (!sv) return CAV_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(job_id);
    if (it == sv->jobs.end()) return CAV_ERR_INVALID_ARGUMENT;
    Job* j = it->second;
    if (j->state == CAV_JOB_PENDING) {  // never admitted: it leaves the queue now
        auto q = std::find(sv->pending.begin(), sv->pending.end(), j);
        if (q != sv->pending.end()) sv->pending.erase(q);
        auto r = std::find(sv->to_parse.begin(), sv->to_parse.end(), j);
        if (r != sv->to_parse.end()) sv->to_parse.erase(r);
        j->desc.reset();  // a loader that is parsing it drops it when done
        j->state = CAV_JOB_CANCELLED;
        j->status = CAV_ERR_CANCELLED;
        j->t_done = sv->now();
        sv->done_cv.notify_all();
    } else if (j->state == CAV_JOB_RUNNING) {  // its lane frees it before its next bounce
        j->cancel = true;
        sv->cv.notify_all();
    }
    return CAV_OK;  // a finished job stays finished
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
    auto pred = [&] {
        return j->state == CAV_JOB_DONE || j->state == CAV_JOB_FAILED || j->state == CAV_JOB_CANCELLED;
    };
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
    out->live = sv->live_count_locked();
    out->hbm_in_use = (int64_t)sv->used;
    return CAV_OK;
}

}  // extern "C"
