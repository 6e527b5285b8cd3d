// Serving loop: continuous batching of all-pairs NW jobs on one device.
//
// Clients submit jobs (sequences + table) from any thread. A worker thread
// owns a context and:
//   * admits queued jobs in arrival order while their device footprint fits
//     the HBM budget and a job slot is free: uploads the sequences, builds
//     their score profiles and allocates the job's output triangle, all kept
//     on the device until the job completes;
//   * launches one merged persistent kernel per quantum, whose task list
//     takes column groups round-robin from every admitted job, so work of a
//     job that arrived while others were running shares the launch with them;
//   * after each launch, finishes jobs whose last task ran (copies the scores
//     out, frees the job's device memory) and admits more.
// Jobs containing sequences that need the reference's orientation (END units
// inside a sequence, GAP units, a non-symmetric table) are scored at
// admission by the single-job path on the same context.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "msa_internal.hpp"

namespace msa {
namespace {

double now_ms()
{
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Job {
    uint64_t id = 0;
    uint32_t n = 0;
    ExtTable ext{};
    msa_table table{};
    std::vector<uint8_t> units;
    std::vector<uint64_t> offs, lens;
    double t_submit = 0, t_admit = 0, t_done = 0;
    uint64_t cells = 0;
    uint32_t launches = 0;
    // device state while admitted
    SeqStore *st = nullptr;
    DevBuf mem;
    int8_t *d_prof = nullptr;
    uint8_t *d_narrow = nullptr;
    int32_t *d_out = nullptr;
    uint64_t device_bytes = 0;
    std::vector<uint32_t> groups;   // column groups per rows pair
    uint32_t cur_k = 0, cur_g = 0;  // next task
    uint64_t total_tasks = 0, issued = 0, finished = 0;
    // result
    std::vector<int32_t> result;
    int status = MSA_OK;
    bool done = false;
};

}  // namespace
}  // namespace msa

struct msa_server {
    msa_ctx *ctx = nullptr;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<msa::Job *> pending;
    std::vector<msa::Job *> admitted;
    std::map<uint64_t, msa::Job *> jobs;
    bool stop = false;
    uint64_t next_id = 1;
    uint64_t budget = 0, used = 0;
    uint32_t max_jobs = 64, quantum = 0;
    double t0 = 0;
    // launch resources (worker thread only)
    msa::DevBuf bound, tasks, views, counter;
    uint64_t bound_stride = 0, grid = 0;
    std::vector<uint32_t> h_tasks;
    std::vector<uint8_t> h_views;
};

namespace msa {
namespace {

constexpr msa::Tiles kServeTiles{32, 8};

// Admits a job. Sets *completed when the job was scored right away (the
// reference-orientation path); the caller publishes completion under the lock.
int admit_one(msa_server *srv, Job *j, bool *completed)
{
    *completed = false;
    msa_ctx *ctx = srv->ctx;
    j->t_admit = now_ms();
    int rc = build_store(ctx, j->units.data(), j->offs.data(), j->lens.data(), j->n, &j->st);
    if(rc) return rc;
    SeqStore *st = j->st;
    unsigned __int128 s1 = 0, s2 = 0;
    for(uint32_t i = 0; i < j->n; ++i) { s1 += j->lens[i]; s2 += (unsigned __int128) j->lens[i] * j->lens[i]; }
    j->cells = (uint64_t) ((s1 * s1 - s2) / 2);
    const uint64_t npairs = (uint64_t) j->n * (j->n - 1) / 2;
    bool symmetric = true;
    for(int x = 0; x < 25 && symmetric; ++x)
        for(int y = 0; y < 25; ++y)
            if(j->ext.score[x * kAlpha + y] != j->ext.score[y * kAlpha + x]) { symmetric = false; break; }
    bool any_dirty = false;
    for(uint32_t i = 0; i < j->n; ++i) any_dirty |= st->dirty[i] != 0;
    j->result.assign(npairs, 0);
    if(any_dirty || !symmetric || j->n < 2) {
        // Reference-orientation path on the same context, synchronously.
        if(j->n >= 2) {
            DevBuf out;
            cudaError_t e = out.ensure(npairs * 4);
            if(e) return cuda_error(ctx, e, "job output");
            std::vector<uint8_t> saved_dirty = st->dirty;
            std::vector<uint32_t> saved_sorted = st->clean_sorted;
            if(!symmetric) {
                std::fill(st->dirty.begin(), st->dirty.end(), 1);
                st->clean_sorted.clear();
            }
            rc = nw_run(ctx, st, j->ext, MSA_NW_PERSISTENT, (int32_t *) out.ptr);
            st->dirty = saved_dirty;
            st->clean_sorted = saved_sorted;
            if(!rc) {
                e = cudaMemcpyAsync(j->result.data(), out.ptr, npairs * 4, cudaMemcpyDeviceToHost, ctx->stream);
                if(!e) e = cudaStreamSynchronize(ctx->stream);
                if(e) rc = cuda_error(ctx, e, "job scores to host");
            }
            drop_plans_for_store(ctx, st->serial);
            out.release();
            j->launches = 1;
        }
        destroy_store(st);
        j->st = nullptr;
        j->t_done = now_ms();
        j->status = rc;
        *completed = true;
        return MSA_OK;   // completed at admission (status carries any error)
    }
    // Resident job: profiles, 16-bit flags, output triangle.
    std::vector<uint8_t> narrow;
    plan_rows_pairs(st, j->ext, kServeTiles, narrow, j->groups);
    const uint32_t K = (uint32_t) narrow.size();
    j->total_tasks = 0;
    for(uint32_t g : j->groups) j->total_tasks += g;
    size_t off = 0;
    auto take = [&off](size_t b) { size_t o = off; off = round_up(off + b, 256); return o; };
    const size_t o_prof = take(st->prof_bytes + 64), o_ext = take(kAlpha * kAlpha), o_nar = take(K + 16),
                 o_out = take(npairs * 4);
    cudaError_t e = j->mem.ensure(off);
    if(e) return cuda_error(ctx, e, "job device memory");
    char *base = (char *) j->mem.ptr;
    j->d_prof = (int8_t *) (base + o_prof);
    j->d_narrow = (uint8_t *) (base + o_nar);
    j->d_out = (int32_t *) (base + o_out);
    e = cudaMemcpyAsync(base + o_ext, j->ext.score, kAlpha * kAlpha, cudaMemcpyHostToDevice, ctx->stream);
    if(!e && K) e = cudaMemcpyAsync(j->d_narrow, narrow.data(), K, cudaMemcpyHostToDevice, ctx->stream);
    if(!e) e = launch_profiles(st, (const int8_t *) (base + o_ext), j->d_prof, ctx->stream);
    if(!e) e = cudaStreamSynchronize(ctx->stream);
    if(e) return cuda_error(ctx, e, "job admission");
    ctx->launches++;
    return MSA_OK;
}

uint64_t estimate_bytes(const Job *j)
{
    uint64_t units = 0, prof = 0;
    for(uint32_t i = 0; i < j->n; ++i) {
        units += round_up(j->lens[i] + 2 + kUnitPad, 16);
        prof += (uint64_t) kAlpha * round_up(std::max<uint64_t>(j->lens[i], 1), kProfPad);
    }
    return units + prof + (uint64_t) j->n * (j->n > 0 ? j->n - 1 : 0) * 2 + (uint64_t) j->n * 40 + 4096;
}

void release_job_device(Job *j)
{
    if(j->st) { destroy_store(j->st); j->st = nullptr; }
    j->mem.release();
}

void worker_loop(msa_server *srv)
{
    msa_ctx *ctx = srv->ctx;
    cudaSetDevice(ctx->device);
    for(;;) {
        // 1. Admission.
        std::vector<Job *> to_admit;
        {
            std::unique_lock<std::mutex> lk(srv->mu);
            if(srv->stop) break;
            while(!srv->pending.empty() && srv->admitted.size() + to_admit.size() < srv->max_jobs) {
                Job *j = srv->pending.front();
                const uint64_t need = estimate_bytes(j);
                if(srv->used + need > srv->budget && !(srv->admitted.empty() && to_admit.empty())) break;
                srv->pending.pop_front();
                j->device_bytes = need;
                srv->used += need;
                to_admit.push_back(j);
            }
            if(to_admit.empty() && srv->admitted.empty()) {
                srv->cv_work.wait_for(lk, std::chrono::milliseconds(20));
                continue;
            }
        }
        for(Job *j : to_admit) {
            bool completed = false;
            const int rc = admit_one(srv, j, &completed);
            if(rc || completed) {
                if(rc) { j->status = rc; j->t_done = now_ms(); }
                release_job_device(j);
            }
            std::lock_guard<std::mutex> lk(srv->mu);
            if(rc || completed) {
                srv->used -= j->device_bytes;
                j->done = true;
                srv->cv_done.notify_all();
            } else {
                srv->admitted.push_back(j);
            }
        }
        std::vector<Job *> active;
        {
            std::lock_guard<std::mutex> lk(srv->mu);
            for(Job *j : srv->admitted) if(j->issued < j->total_tasks) active.push_back(j);
        }
        if(active.empty()) continue;

        // 2. One merged launch: column groups round-robin over the admitted jobs.
        uint64_t max_cols = 1;
        for(Job *j : active) for(uint32_t i = 0; i < j->n; ++i) max_cols = std::max<uint64_t>(max_cols, j->st->plen[i]);
        const uint64_t stride = round_up(max_cols + 160, 32);
        if(!srv->grid && serve_grid(ctx, &srv->grid)) break;
        if(stride > srv->bound_stride) {
            if(srv->bound.ensure(srv->grid * kServeTiles.W * stride * 4)) break;
            srv->bound_stride = stride;
        }
        const uint64_t quantum = srv->quantum ? srv->quantum : 4 * srv->grid;
        srv->h_tasks.clear();
        const size_t vb = job_view_bytes();
        srv->h_views.assign(active.size() * vb, 0);
        std::vector<uint64_t> taken(active.size(), 0);
        for(size_t s = 0; s < active.size(); ++s)
            fill_job_view(srv->h_views.data() + s * vb, active[s]->st, active[s]->d_prof, active[s]->d_narrow,
                          active[s]->d_out, active[s]->ext.penalty);
        bool any = true;
        while(srv->h_tasks.size() / 4 < quantum && any) {
            any = false;
            for(size_t s = 0; s < active.size() && srv->h_tasks.size() / 4 < quantum; ++s) {
                Job *j = active[s];
                if(j->issued + taken[s] >= j->total_tasks) continue;
                // advance the job's cursor to its next (rows pair, group)
                while(j->cur_k < j->groups.size() && j->cur_g >= j->groups[j->cur_k]) { ++j->cur_k; j->cur_g = 0; }
                srv->h_tasks.push_back((uint32_t) s);
                srv->h_tasks.push_back(j->cur_k);
                srv->h_tasks.push_back(j->cur_g);
                srv->h_tasks.push_back(0);
                ++j->cur_g;
                ++taken[s];
                any = true;
            }
        }
        const uint64_t ntasks = srv->h_tasks.size() / 4;
        cudaError_t e = srv->tasks.ensure(ntasks * 16 + 16);
        if(!e) e = srv->views.ensure(srv->h_views.size() + 16);
        if(!e) e = srv->counter.ensure(64);
        if(!e) e = cudaMemcpyAsync(srv->tasks.ptr, srv->h_tasks.data(), ntasks * 16, cudaMemcpyHostToDevice, ctx->stream);
        if(!e) e = cudaMemcpyAsync(srv->views.ptr, srv->h_views.data(), srv->h_views.size(), cudaMemcpyHostToDevice,
                                   ctx->stream);
        if(!e) e = cudaMemsetAsync(srv->counter.ptr, 0, 64, ctx->stream);
        if(!e) {
            ServeLaunch L{srv->views.ptr, srv->tasks.ptr, ntasks, (uint32_t *) srv->bound.ptr, srv->bound_stride,
                          (unsigned long long *) srv->counter.ptr};
            e = launch_serve(L, srv->grid, ctx->stream);
            ctx->launches++;
        }
        if(!e) e = cudaStreamSynchronize(ctx->stream);
        const bool failed = e != cudaSuccess;
        if(failed) cuda_error(ctx, e, "serving launch");

        // 3. Account; finish jobs whose last task ran (device memory released
        // before completion is published under the lock).
        std::vector<Job *> finished;
        for(size_t s = 0; s < active.size(); ++s) {
            Job *j = active[s];
            j->issued += taken[s];
            j->finished += taken[s];
            if(taken[s]) ++j->launches;
            if(failed) {
                j->status = MSA_ERR_CUDA;
            } else if(j->finished >= j->total_tasks) {
                const uint64_t npairs = (uint64_t) j->n * (j->n - 1) / 2;
                cudaError_t e2 = cudaMemcpyAsync(j->result.data(), j->d_out, npairs * 4, cudaMemcpyDeviceToHost,
                                                 ctx->stream);
                if(!e2) e2 = cudaStreamSynchronize(ctx->stream);
                j->status = e2 ? cuda_error(ctx, e2, "job scores to host") : MSA_OK;
            } else {
                continue;
            }
            j->t_done = now_ms();
            release_job_device(j);
            finished.push_back(j);
        }
        if(!finished.empty()) {
            std::lock_guard<std::mutex> lk(srv->mu);
            auto &adm = srv->admitted;
            for(Job *j : finished) {
                srv->used -= j->device_bytes;
                adm.erase(std::find(adm.begin(), adm.end(), j));
                j->done = true;
            }
            srv->cv_done.notify_all();
        }
    }
    // Stopping: fail what is still queued or admitted.
    std::lock_guard<std::mutex> lk(srv->mu);
    for(Job *j : srv->pending) { j->status = MSA_ERR_QUEUE; j->done = true; }
    srv->pending.clear();
    for(Job *j : srv->admitted) { release_job_device(j); j->status = MSA_ERR_QUEUE; j->done = true; }
    srv->admitted.clear();
    srv->cv_done.notify_all();
}

}  // namespace
}  // namespace msa

using namespace msa;

extern "C" {

int msa_serve_start(const msa_serve_config *cfg, msa_server **out)
{
    if(!cfg || !out) return MSA_ERR_INVALID;
    *out = nullptr;
    msa_server *srv = nullptr;
    try {
        srv = new msa_server;
        int rc = msa_create(cfg->device, &srv->ctx);
        if(rc) { delete srv; return rc; }
        size_t free_b = 0, total_b = 0;
        cudaSetDevice(cfg->device);
        if(cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) { cudaGetLastError(); free_b = 0; }
        srv->budget = cfg->hbm_budget_bytes ? cfg->hbm_budget_bytes : (uint64_t) (0.8 * (double) free_b);
        srv->max_jobs = cfg->max_jobs ? cfg->max_jobs : 64;
        srv->quantum = cfg->quantum_pairs;
        srv->t0 = now_ms();
        srv->worker = std::thread(worker_loop, srv);
        *out = srv;
        return MSA_OK;
    } catch(...) {
        if(srv) {
            if(srv->ctx) msa_destroy(srv->ctx);
            delete srv;
        }
        return MSA_ERR_NOMEM;
    }
}

int msa_serve_submit(msa_server *srv, const uint8_t *units, const uint64_t *offs, const uint64_t *lens, uint32_t n,
                     const msa_table *table, uint64_t *job_id)
{
    if(!srv || !table || !job_id || (n && (!offs || !lens))) return MSA_ERR_INVALID;
    try {
        Job *j = new Job;
        j->n = n;
        j->table = *table;
        std::string err;
        const int rc = make_ext_table(table, &j->ext, &err);
        if(rc) { delete j; return rc; }
        uint64_t total = 0;
        for(uint32_t i = 0; i < n; ++i) total += lens[i];
        j->units.resize(total);
        j->offs.resize(n);
        j->lens.assign(lens, lens + n);
        uint64_t pos = 0;
        for(uint32_t i = 0; i < n; ++i) {
            if(lens[i] && !units) { delete j; return MSA_ERR_INVALID; }
            if(lens[i]) std::memcpy(j->units.data() + pos, units + offs[i], lens[i]);
            j->offs[i] = pos;
            pos += lens[i];
        }
        for(uint8_t u : j->units) if(u > MSA_UNIT_GAP) { delete j; return MSA_ERR_INVALID; }
        std::lock_guard<std::mutex> lk(srv->mu);
        if(srv->stop) { delete j; return MSA_ERR_QUEUE; }
        j->id = srv->next_id++;
        j->t_submit = now_ms();
        srv->jobs[j->id] = j;
        srv->pending.push_back(j);
        *job_id = j->id;
        srv->cv_work.notify_one();
        return MSA_OK;
    } catch(...) {
        return MSA_ERR_NOMEM;
    }
}

int msa_serve_wait(msa_server *srv, uint64_t job_id, int timeout_ms, int32_t *out, msa_job_stats *stats)
{
    if(!srv) return MSA_ERR_INVALID;
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->jobs.find(job_id);
    if(it == srv->jobs.end()) return MSA_ERR_QUEUE;
    Job *j = it->second;
    auto ready = [j]() { return j->done; };
    if(timeout_ms < 0) srv->cv_done.wait(lk, ready);
    else if(!srv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return MSA_ERR_DEVICE_TIMEOUT;
    const int status = j->status;
    if(out && !j->result.empty()) std::memcpy(out, j->result.data(), j->result.size() * 4);
    if(stats) {
        stats->submit_ms = j->t_submit - srv->t0;
        stats->admit_ms = j->t_admit - srv->t0;
        stats->done_ms = j->t_done - srv->t0;
        stats->cells = j->cells;
        stats->n = j->n;
        stats->launches = j->launches;
    }
    srv->jobs.erase(it);
    delete j;
    return status;
}

int msa_serve_stop(msa_server *srv)
{
    if(!srv) return MSA_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stop = true;
        srv->cv_work.notify_all();
    }
    if(srv->worker.joinable()) srv->worker.join();
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        for(auto &kv : srv->jobs) delete kv.second;
        srv->jobs.clear();
    }
    cudaSetDevice(srv->ctx->device);
    srv->bound.release();
    srv->tasks.release();
    srv->views.release();
    srv->counter.release();
    msa_destroy(srv->ctx);
    delete srv;
    return MSA_OK;
}

}  // extern "C"
