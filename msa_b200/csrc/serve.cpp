// Serving loop: continuous batching of all-pairs NW jobs on one device.
//
// Clients submit jobs (sequences + table) from any thread. Two threads, each
// with its own context and stream, serve them:
//   * the admission thread takes queued jobs in arrival order while their
//     device footprint fits the HBM budget and a job slot is free: uploads
//     the sequences, builds their score profiles and allocates the job's
//     output triangle, all kept on the device until the job completes;
//   * the launch thread issues one merged persistent kernel per quantum,
//     whose task list takes column groups from every admitted job, so work of
//     a job that arrived while others were running shares the launch with
//     them; two launches are kept in flight on two streams (each with its own
//     boundary rows and task tables, so the second fills the SMs the first
//     one's last tasks leave idle), and after each one the jobs whose last
//     task ran are finished (scores copied out, device memory returned).
// Job memory comes from a memory pool of the server in stream order, so
// neither admission nor release waits for the launches in flight. The launch
// thread returns memory on a stream of its own: the admission stream may be
// capturing a CUDA graph, which would absorb a release enqueued there.
// msa_serve_start pays the one-time costs (pool growth, launch buffers, pinned
// staging, a first launch on no work) before the server takes jobs.
//
// Two policies share the quantum's cell budget among the admitted jobs:
//   * continuous (batch_window_us = 0): every job gets an equal share, so a
//     job's latency is about its own work times the number of jobs sharing the
//     device; with age_weight_us = A > 0 the shares are weighted by
//     1 + age / A instead, which moves budget to the jobs that have waited
//     longest;
//   * batch windows (batch_window_us = W): a job submitted in window k (from
//     server start) is admitted at the window's end, the windows are served in
//     order (older windows take the budget first), and inside a window the
//     budget is split in proportion to each job's remaining cells, so the jobs
//     of a window advance together and finish in the same quantum. Latency is
//     then close to the window's wait plus the window's work, whatever the
//     job's own size.
// Jobs containing sequences that need the reference's orientation (END units
// inside a sequence, GAP units, a non-symmetric table) are recognised on the
// host at admission and handed to a third thread with its own context and
// stream, which scores them one at a time by the single-job path; admission
// and the merged launches never wait for them.
#include <algorithm>
#include <cmath>
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
    uint64_t window = 0;            // admission window index (batch windows)
    // device state while admitted
    SeqStore *st = nullptr;
    void *mem = nullptr;            // profiles, flags, table, output (pooled)
    int8_t *d_prof = nullptr;
    uint8_t *d_narrow = nullptr;
    int32_t *d_out = nullptr;
    uint64_t device_bytes = 0;
    std::vector<uint32_t> groups;   // column groups per rows pair
    std::vector<uint8_t> narrow;    // 16-bit flag per rows pair (host copy)
    const int8_t *d_ext = nullptr;  // extended table on the device
    uint32_t cur_k = 0, cur_g = 0;  // next task
    uint64_t total_tasks = 0, issued = 0, finished = 0;
    uint64_t tcells_total = 0, tcells_issued = 0;   // estimated cells of all / issued tasks
    // result
    std::vector<int32_t> result;
    int status = MSA_OK;
    bool done = false;
};

}  // namespace
}  // namespace msa

struct msa_server {
    msa_ctx *ctx = nullptr;   // launch thread
    msa_ctx *adm = nullptr;   // admission thread
    msa_ctx *ori = nullptr;   // reference-orientation thread
    cudaMemPool_t pool = nullptr;
    cudaStream_t adm_stream = nullptr;   // highest-priority stream of the admission context
    std::thread worker, admitter, orienter;
    std::mutex mu;
    std::condition_variable cv_work, cv_launch, cv_done, cv_oriented;
    std::deque<msa::Job *> pending;
    std::deque<msa::Job *> oriented;   // admitted jobs for the reference-orientation thread
    std::vector<msa::Job *> admitted;
    std::map<uint64_t, msa::Job *> jobs;
    bool stop = false;
    bool worker_ready = false;   // the launch thread has its staging buffers
    uint64_t next_id = 1;
    uint64_t budget = 0, used = 0;
    uint32_t max_jobs = 64, quantum = 0;
    double window_ms = 0;   // admission window (0 = admit at once)
    double age_ms = 0;      // continuous admission: share weight 1 + age / age_ms (0 = equal shares)
    double t0 = 0;
    // launch resources (worker thread only)
    msa::DevBuf bound, tasks, views, counter, bound2, tasks2, views2, counter2;
    uint64_t bound_stride = 0, grid = 0;
    std::vector<uint32_t> h_tasks;
    std::vector<uint8_t> h_views;
};

namespace msa {
namespace {

constexpr msa::Tiles kServeTiles{32, 8};

// Estimated cells of task (rows pair k, group g) of a job.
static uint64_t task_cells(const Job *j, uint32_t k, uint32_t g)
{
    const SeqStore *st = j->st;
    const uint32_t nclean = (uint32_t) st->clean_sorted.size();
    const uint64_t e1 = st->eff[st->clean_sorted[2 * k]];
    const uint32_t b0 = 2 * k + 1 + g * kServeTiles.W;
    const uint32_t bn = std::min<uint32_t>(nclean, b0 + kServeTiles.W);
    const uint64_t c0 = b0 < nclean ? st->eff[st->clean_sorted[b0]] : 0;
    return 2 * e1 * c0 * (bn > b0 ? bn - b0 : 0);
}

// Whether a job needs the reference's orientation (the single-job path):
// a sequence with END units before its last letter, an empty one or one with
// GAP units (the store's "dirty" rule, scan_units), a table that is not
// symmetric, or fewer than two sequences. Decided on the host from the job's
// units.
bool needs_reference_orientation(const Job *j)
{
    if(j->n < 2) return true;
    for(int x = 0; x < 25; ++x)
        for(int y = 0; y < 25; ++y)
            if(j->ext.score[x * kAlpha + y] != j->ext.score[y * kAlpha + x]) return true;
    for(uint32_t i = 0; i < j->n; ++i) {
        const uint32_t plen = (uint32_t) ((j->lens[i] + 2) / 3 * 3);
        uint32_t eff = 0;
        uint8_t dirty = 0, gap = 0;
        scan_units(j->units.data() + j->offs[i], j->lens[i], plen, &eff, &dirty, &gap);
        if(dirty) return true;
    }
    return false;
}

uint64_t job_cells(const Job *j)
{
    unsigned __int128 s1 = 0, s2 = 0;
    for(uint32_t i = 0; i < j->n; ++i) { s1 += j->lens[i]; s2 += (unsigned __int128) j->lens[i] * j->lens[i]; }
    return (uint64_t) ((s1 * s1 - s2) / 2);
}

// Scores a job in the reference's orientation on the reference-orientation
// context, synchronously (msa_nw_all_pairs's path: nw_run with every pair of
// a dirty sequence, or every pair under a non-symmetric table, in the
// reference's orientation). Device memory comes from the server's pool on
// that context's stream and is returned there once the scores are on the host.
int score_oriented(msa_server *srv, Job *j)
{
    msa_ctx *ctx = srv->ori;
    j->cells = job_cells(j);
    const uint64_t npairs = (uint64_t) j->n * (j->n > 0 ? j->n - 1 : 0) / 2;
    j->result.assign(npairs, 0);
    if(j->n < 2) return MSA_OK;
    SeqStore *st = nullptr;
    int rc = build_store(ctx, j->units.data(), j->offs.data(), j->lens.data(), j->n, &st);
    if(rc) return rc;
    bool symmetric = true;
    for(int x = 0; x < 25 && symmetric; ++x)
        for(int y = 0; y < 25; ++y)
            if(j->ext.score[x * kAlpha + y] != j->ext.score[y * kAlpha + x]) { symmetric = false; break; }
    if(!symmetric) {
        std::fill(st->dirty.begin(), st->dirty.end(), 1);
        st->clean_sorted.clear();
    }
    void *out = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&out, npairs * 4, srv->pool, ctx->stream);
    if(e) {
        destroy_store_async(st, ctx->stream);
        return cuda_error(ctx, e, "job output");
    }
    rc = nw_run(ctx, st, j->ext, MSA_NW_PERSISTENT, (int32_t *) out);
    if(!rc) {
        e = cudaMemcpyAsync(j->result.data(), out, npairs * 4, cudaMemcpyDeviceToHost, ctx->stream);
        if(!e) e = cudaStreamSynchronize(ctx->stream);
        if(e) rc = cuda_error(ctx, e, "job scores to host");
    }
    drop_plans_for_store(ctx, st->serial);
    cudaFreeAsync(out, ctx->stream);
    destroy_store_async(st, ctx->stream);
    j->launches = 1;
    return rc;
}

// Reference-orientation thread: scores the jobs admission handed over, one at
// a time, and publishes each completion.
void orientation_loop(msa_server *srv)
{
    cudaSetDevice(srv->ori->device);
    for(;;) {
        Job *j = nullptr;
        {
            std::unique_lock<std::mutex> lk(srv->mu);
            srv->cv_oriented.wait(lk, [srv] { return srv->stop || !srv->oriented.empty(); });
            if(srv->stop) return;
            j = srv->oriented.front();
            srv->oriented.pop_front();
        }
        j->t_admit = now_ms();
        const int rc = score_oriented(srv, j);
        std::lock_guard<std::mutex> lk(srv->mu);
        j->status = rc;
        j->t_done = now_ms();
        j->done = true;
        srv->used -= j->device_bytes;
        srv->cv_done.notify_all();
        srv->cv_work.notify_all();
    }
}

// Admits a resident job on the admission context: uploads its sequences,
// table and flags and allocates its output (the score profiles are left to
// launch_job_profiles, so that the uploads of a batch of jobs do not queue
// behind one another's kernels). The job holds clean sequences only and a
// symmetric table (needs_reference_orientation is false).
int admit_one(msa_server *srv, Job *j)
{
    msa_ctx *ctx = srv->adm;
    j->t_admit = now_ms();
    int rc = build_store(ctx, j->units.data(), j->offs.data(), j->lens.data(), j->n, &j->st);
    if(rc) return rc;
    SeqStore *st = j->st;
    j->cells = job_cells(j);
    const uint64_t npairs = (uint64_t) j->n * (j->n - 1) / 2;
    j->result.assign(npairs, 0);
    // Resident job: profiles, 16-bit flags, output triangle.
    plan_rows_pairs(st, j->ext, kServeTiles, j->narrow, j->groups);
    const uint32_t K = (uint32_t) j->narrow.size();
    j->total_tasks = 0;
    j->tcells_total = 0;
    for(uint32_t k = 0; k < (uint32_t) j->groups.size(); ++k) {
        j->total_tasks += j->groups[k];
        for(uint32_t g = 0; g < j->groups[k]; ++g) j->tcells_total += task_cells(j, k, g);
    }
    size_t off = 0;
    auto take = [&off](size_t b) { size_t o = off; off = round_up(off + b, 256); return o; };
    const size_t o_prof = take(st->prof_bytes + 64), o_ext = take(kAlpha * kAlpha), o_nar = take(K + 16),
                 o_out = take(npairs * 4);
    cudaError_t e = cudaMallocFromPoolAsync(&j->mem, off, srv->pool, ctx->stream);
    if(e) { j->mem = nullptr; return cuda_error(ctx, e, "job device memory"); }
    char *base = (char *) j->mem;
    j->d_prof = (int8_t *) (base + o_prof);
    j->d_narrow = (uint8_t *) (base + o_nar);
    j->d_out = (int32_t *) (base + o_out);
    j->d_ext = (const int8_t *) (base + o_ext);
    e = cudaMemcpyAsync(base + o_ext, j->ext.score, kAlpha * kAlpha, cudaMemcpyHostToDevice, ctx->stream);
    if(!e && K) e = cudaMemcpyAsync(j->d_narrow, j->narrow.data(), K, cudaMemcpyHostToDevice, ctx->stream);
    if(e) return cuda_error(ctx, e, "job admission");
    return MSA_OK;
}

// Score profiles of an admitted resident job, on the admission stream.
int launch_job_profiles(msa_server *srv, Job *j)
{
    msa_ctx *ctx = srv->adm;
    const cudaError_t e = launch_profiles(j->st, j->d_ext, j->d_prof, ctx->stream);
    if(e) return cuda_error(ctx, e, "job profiles");
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

// Returns a job's device memory to the pool in stream order on `s` (the
// job's last launch has completed, or it never ran).
void release_job_device(Job *j, cudaStream_t s)
{
    if(j->st) { destroy_store_async(j->st, s); j->st = nullptr; }
    if(j->mem) { cudaFreeAsync(j->mem, s); j->mem = nullptr; }
}

// One launch in flight: its completion event and the tasks it took per job.
struct InFlight {
    cudaEvent_t done = nullptr;
    std::vector<std::pair<Job *, uint64_t>> work;
    bool busy = false;
    // Pinned staging for this slot's task list and job table (rewritten only
    // after the slot's previous launch, which consumed them, has retired).
    void *h_tasks = nullptr, *h_views = nullptr;
    size_t tasks_cap = 0, views_cap = 0;
    bool stage(size_t tb, size_t vbytes)
    {
        if(tb > tasks_cap) {
            if(h_tasks) cudaFreeHost(h_tasks);
            tasks_cap = std::max(tb, tasks_cap * 2);
            if(cudaMallocHost(&h_tasks, tasks_cap) != cudaSuccess) { h_tasks = nullptr; tasks_cap = 0; return false; }
        }
        if(vbytes > views_cap) {
            if(h_views) cudaFreeHost(h_views);
            views_cap = std::max(vbytes, views_cap * 2);
            if(cudaMallocHost(&h_views, views_cap) != cudaSuccess) { h_views = nullptr; views_cap = 0; return false; }
        }
        return true;
    }
    void release()
    {
        if(h_tasks) cudaFreeHost(h_tasks);
        if(h_views) cudaFreeHost(h_views);
        h_tasks = h_views = nullptr;
        tasks_cap = views_cap = 0;
    }
};

// Admission thread: takes queued jobs in arrival order (at their window's
// end under batch windows) while the HBM budget and the job slots allow, and
// hands them to the launch thread. All jobs eligible at once are admitted as
// one batch: their uploads first, then their profile kernels, then a single
// wait. The admission stream has the device's highest priority, so these
// kernels take SMs at the next boundary of the merged launches.
void admission_loop(msa_server *srv)
{
    msa_ctx *ctx = srv->adm;
    cudaSetDevice(ctx->device);
    for(;;) {
        std::vector<Job *> batch;
        {
            std::unique_lock<std::mutex> lk(srv->mu);
            for(;;) {
                if(srv->stop) return;
                double wait_ms = 20.0;
                const double now = now_ms();
                while(!srv->pending.empty() && srv->admitted.size() + batch.size() < srv->max_jobs) {
                    Job *f = srv->pending.front();
                    const double gate = srv->window_ms > 0 ? srv->t0 + (double) f->window * srv->window_ms : 0.0;
                    if(now < gate) {
                        wait_ms = std::max(0.05, std::min(wait_ms, gate - now));
                        break;
                    }
                    const uint64_t need = estimate_bytes(f);
                    // A job larger than the whole budget is admitted alone.
                    if(srv->used + need > srv->budget && !(srv->admitted.empty() && batch.empty())) break;
                    srv->pending.pop_front();
                    f->device_bytes = need;
                    srv->used += need;
                    batch.push_back(f);
                }
                if(!batch.empty()) break;
                srv->cv_work.wait_for(lk, std::chrono::microseconds((long long) (wait_ms * 1000)));
            }
        }
        // Jobs for the single-job path go to the reference-orientation thread
        // (with their memory reservation) without touching the device here.
        {
            std::vector<Job *> resident;
            bool handed = false;
            for(Job *j : batch) {
                if(needs_reference_orientation(j)) {
                    std::lock_guard<std::mutex> lk(srv->mu);
                    srv->oriented.push_back(j);
                    handed = true;
                } else {
                    resident.push_back(j);
                }
            }
            if(handed) srv->cv_oriented.notify_one();
            batch.swap(resident);
            if(batch.empty()) continue;
        }
        std::vector<int> status(batch.size(), MSA_OK);
        for(size_t i = 0; i < batch.size(); ++i) status[i] = admit_one(srv, batch[i]);
        for(size_t i = 0; i < batch.size(); ++i)
            if(!status[i]) status[i] = launch_job_profiles(srv, batch[i]);
        const cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if(e) {
            const int rc = cuda_error(ctx, e, "job admission");
            for(size_t i = 0; i < batch.size(); ++i) if(!status[i]) status[i] = rc;
        }
        for(size_t i = 0; i < batch.size(); ++i) {
            Job *j = batch[i];
            if(status[i]) {
                j->status = status[i];
                j->t_done = now_ms();
                release_job_device(j, ctx->stream);
            }
        }
        std::lock_guard<std::mutex> lk(srv->mu);
        bool any = false;
        for(size_t i = 0; i < batch.size(); ++i) {
            Job *j = batch[i];
            if(status[i]) {
                srv->used -= j->device_bytes;
                j->done = true;
            } else {
                srv->admitted.push_back(j);
                any = true;
            }
        }
        srv->cv_done.notify_all();
        if(any) srv->cv_launch.notify_one();
    }
}

// Launch thread: merged launches over the admitted jobs, two in flight.
void worker_loop(msa_server *srv)
{
    msa_ctx *ctx = srv->ctx;
    cudaSetDevice(ctx->device);
    // The two launches in flight run on two streams with their own boundary
    // rows, so the next launch's CTAs fill the SMs that the previous launch's
    // last tasks leave idle. Their tasks are disjoint pairs.
    cudaStream_t compute2 = nullptr, drain = nullptr;
    cudaStreamCreateWithFlags(&compute2, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&drain, cudaStreamNonBlocking);
    const cudaStream_t slot_stream[2] = {ctx->own_stream, compute2};
    // Job memory goes back to the pool on this thread's own copy stream, never
    // on another thread's stream: the reference-orientation thread may be
    // capturing a CUDA graph on its stream, and a free enqueued on a capturing
    // stream would become part of that graph. The pool hands the memory to the
    // next admissions once the free has completed.
    const cudaStream_t release_stream = drain;
    InFlight slots[2];
    for(auto &f : slots) {
        cudaEventCreateWithFlags(&f.done, cudaEventDisableTiming);
        f.stage(1 << 20, 64 << 10);   // pinned staging before the first job
    }
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->worker_ready = true;
    }
    srv->cv_done.notify_all();
    int cur = 0;
    const size_t vb = job_view_bytes();

    // Applies a completed launch: counts its tasks and finishes jobs whose
    // last task ran (scores copied out, device memory released, completion
    // published under the lock).
    auto retire = [&](InFlight &f) {
        if(!f.busy) return;
        const cudaError_t e = cudaEventSynchronize(f.done);
        std::vector<Job *> finished;
        for(auto &w : f.work) {
            Job *j = w.first;
            j->finished += w.second;
            if(e) j->status = MSA_ERR_CUDA;
            if(j->finished >= j->total_tasks && !j->done) {
                if(!e && j->status == MSA_OK) {
                    const uint64_t npairs = (uint64_t) j->n * (j->n - 1) / 2;
                    cudaError_t e2 = cudaMemcpyAsync(j->result.data(), j->d_out, npairs * 4, cudaMemcpyDeviceToHost, drain);
                    if(!e2) e2 = cudaStreamSynchronize(drain);
                    if(e2) j->status = cuda_error(ctx, e2, "job scores to host");
                }
                j->t_done = now_ms();
                release_job_device(j, release_stream);
                finished.push_back(j);
            }
        }
        if(e) cuda_error(ctx, e, "serving launch");
        f.work.clear();
        f.busy = false;
        if(!finished.empty()) {
            std::lock_guard<std::mutex> lk(srv->mu);
            auto &adm = srv->admitted;
            for(Job *j : finished) {
                srv->used -= j->device_bytes;
                adm.erase(std::find(adm.begin(), adm.end(), j));
                j->done = true;
            }
            srv->cv_done.notify_all();
            srv->cv_work.notify_all();   // memory and job slots are free again
        }
    };

    const uint64_t budget_cells = srv->quantum ? (uint64_t) srv->quantum * 1000000ull : 40000000000ull;
    for(;;) {
        // 1. Retire the launch that used this slot two rounds ago.
        retire(slots[cur]);

        // 2. The admitted jobs with tasks left (in admission order).
        std::vector<Job *> active;
        {
            std::unique_lock<std::mutex> lk(srv->mu);
            if(srv->stop) break;
            for(Job *j : srv->admitted) if(j->issued < j->total_tasks) active.push_back(j);
            if(active.empty() && !slots[cur ^ 1].busy) {
                srv->cv_launch.wait_for(lk, std::chrono::milliseconds(20));
                continue;
            }
        }
        if(active.empty()) {
            retire(slots[cur ^ 1]);
            continue;
        }

        // 3. Each job's cell quota in this launch.
        std::vector<uint64_t> quota(active.size(), 0);
        if(srv->window_ms > 0) {
            // Windows in order; the last window reached splits what is left
            // in proportion to its jobs' remaining cells.
            uint64_t left = budget_cells;
            for(size_t a = 0; a < active.size() && left > 0;) {
                size_t b = a;
                uint64_t rem = 0;
                while(b < active.size() && active[b]->window == active[a]->window) {
                    rem += active[b]->tcells_total - active[b]->tcells_issued;
                    ++b;
                }
                for(size_t i = a; i < b; ++i) {
                    const uint64_t r = active[i]->tcells_total - active[i]->tcells_issued;
                    quota[i] = rem <= left ? ~0ull
                                           : std::max<uint64_t>((uint64_t) ((unsigned __int128) left * r / std::max<uint64_t>(rem, 1)), 1);
                }
                left = rem <= left ? left - rem : 0;
                a = b;
            }
        } else if(srv->age_ms > 0) {
            // Shares weighted by 1 + age / age_ms.
            const double now = now_ms();
            std::vector<double> w(active.size());
            double sum = 0;
            for(size_t i = 0; i < active.size(); ++i) {
                w[i] = 1.0 + std::max(0.0, now - active[i]->t_submit) / srv->age_ms;
                sum += w[i];
            }
            for(size_t i = 0; i < active.size(); ++i)
                quota[i] = std::max<uint64_t>((uint64_t) ((double) budget_cells * w[i] / sum), 1);
        } else {
            std::fill(quota.begin(), quota.end(), std::max<uint64_t>(budget_cells / active.size(), 1));
        }

        // 4. One merged launch: tasks taken in each job's cost order up to its
        // quota, then sorted longest first so the launch's tail holds its
        // smallest tasks.
        uint64_t max_cols = 1;
        for(Job *j : active) for(uint32_t i = 0; i < j->n; ++i) max_cols = std::max<uint64_t>(max_cols, j->st->plen[i]);
        const uint64_t stride = round_up(max_cols + 160, 32);
        if(!srv->grid && serve_grid(ctx, &srv->grid)) break;
        if(stride > srv->bound_stride) {
            retire(slots[cur ^ 1]);   // the buffers are about to move
            const uint64_t bytes = srv->grid * kServeTiles.W * std::max<uint64_t>(stride, 2048 + 160) * 4;
            if(srv->bound.ensure(bytes) || srv->bound2.ensure(bytes)) break;
            srv->bound_stride = std::max<uint64_t>(stride, 2048 + 160);
        }
        struct T { uint32_t slot, k, g; uint64_t cost; };
        std::vector<T> tasks;
        InFlight &f = slots[cur];
        f.work.clear();
        srv->h_views.assign(active.size() * vb, 0);
        for(size_t sl = 0; sl < active.size(); ++sl) {
            Job *j = active[sl];
            fill_job_view(srv->h_views.data() + sl * vb, j->st, j->d_prof, j->d_narrow, j->d_out, j->ext.penalty);
            uint64_t taken = 0, cells = 0;
            while(j->issued + taken < j->total_tasks && cells < quota[sl]) {
                while(j->cur_k < j->groups.size() && j->cur_g >= j->groups[j->cur_k]) { ++j->cur_k; j->cur_g = 0; }
                const uint64_t c = task_cells(j, j->cur_k, j->cur_g);
                tasks.push_back({(uint32_t) sl, j->cur_k, j->cur_g, c});
                cells += c;
                ++j->cur_g;
                ++taken;
            }
            j->issued += taken;
            j->tcells_issued += cells;
            if(taken) { f.work.push_back({j, taken}); ++j->launches; }
        }
        std::stable_sort(tasks.begin(), tasks.end(), [](const T &a, const T &b) { return a.cost > b.cost; });
        const uint64_t ntasks = tasks.size();
        if(!f.stage(ntasks * 16 + 16, srv->h_views.size() + 16)) { cuda_error(ctx, cudaErrorMemoryAllocation, "pinned staging"); break; }
        uint32_t *ht = (uint32_t *) f.h_tasks;
        for(size_t q = 0; q < tasks.size(); ++q) {
            ht[4 * q] = tasks[q].slot;
            ht[4 * q + 1] = tasks[q].k;
            ht[4 * q + 2] = tasks[q].g;
            ht[4 * q + 3] = 0;
        }
        std::memcpy(f.h_views, srv->h_views.data(), srv->h_views.size());
        // Device buffers of this slot: grow only while nothing else is in flight.
        DevBuf &tb = cur ? srv->tasks : srv->tasks2, &vbuf = cur ? srv->views : srv->views2,
               &cb = cur ? srv->counter : srv->counter2, &bb = cur ? srv->bound2 : srv->bound;
        const cudaStream_t compute = slot_stream[cur];
        if(tb.bytes < ntasks * 16 + 16 || vbuf.bytes < srv->h_views.size() + 16) retire(slots[cur ^ 1]);
        cudaError_t e = tb.ensure(std::max<size_t>(ntasks * 16 + 16, 1 << 20));
        if(!e) e = vbuf.ensure(std::max<size_t>(srv->h_views.size() + 16, 64 << 10));
        if(!e) e = cb.ensure(64);
        if(!e) e = cudaMemcpyAsync(tb.ptr, f.h_tasks, ntasks * 16, cudaMemcpyHostToDevice, compute);
        if(!e) e = cudaMemcpyAsync(vbuf.ptr, f.h_views, srv->h_views.size(), cudaMemcpyHostToDevice, compute);
        if(!e) e = cudaMemsetAsync(cb.ptr, 0, 64, compute);
        if(!e) {
            ServeLaunch L{vbuf.ptr, tb.ptr, ntasks, (uint32_t *) bb.ptr, srv->bound_stride,
                          (unsigned long long *) cb.ptr};
            e = launch_serve(L, srv->grid, compute);
            ctx->launches++;
        }
        if(!e) e = cudaEventRecord(f.done, compute);
        if(e) cuda_error(ctx, e, "serving launch");
        f.busy = true;
        cur ^= 1;
    }
    retire(slots[0]);
    retire(slots[1]);
    for(auto &f : slots) { cudaEventDestroy(f.done); f.release(); }
    cudaStreamDestroy(drain);
    cudaStreamDestroy(compute2);
}

// Pays a server's one-time costs before it takes jobs, so that they do not
// fall on the first jobs' latency: the job-memory pool grows to hold up to
// 2 GiB (released memory stays in the pool), both launch slots get their
// boundary rows (sequences up to 2,048 units; longer ones grow them later)
// and task tables, and the serving kernel runs once on an empty task list.
int warm_server(msa_server *srv)
{
    msa_ctx *ctx = srv->ctx;
    cudaSetDevice(ctx->device);
    const uint64_t warm = std::min<uint64_t>(srv->budget, 2ull << 30);
    if(srv->pool && warm) {
        void *p = nullptr;
        cudaError_t e = cudaMallocFromPoolAsync(&p, warm, srv->pool, srv->adm->stream);
        if(!e) e = cudaFreeAsync(p, srv->adm->stream);
        if(!e) e = cudaStreamSynchronize(srv->adm->stream);
        if(e) return cuda_error(srv->adm, e, "job memory pool");
    }
    if(const int rc = serve_grid(ctx, &srv->grid)) return rc;
    const uint64_t stride = 2048 + 160;
    const uint64_t bytes = srv->grid * kServeTiles.W * stride * 4;
    cudaError_t e = srv->bound.ensure(bytes);
    if(!e) e = srv->bound2.ensure(bytes);
    if(!e) e = srv->tasks.ensure(1 << 20);
    if(!e) e = srv->tasks2.ensure(1 << 20);
    if(!e) e = srv->views.ensure(64 << 10);
    if(!e) e = srv->views2.ensure(64 << 10);
    if(!e) e = srv->counter.ensure(64);
    if(!e) e = srv->counter2.ensure(64);
    if(e) return cuda_error(ctx, e, "serving buffers");
    srv->bound_stride = stride;
    e = cudaMemsetAsync(srv->counter.ptr, 0, 64, ctx->own_stream);
    const ServeLaunch L{srv->views.ptr, srv->tasks.ptr, 0, (uint32_t *) srv->bound.ptr, stride,
                        (unsigned long long *) srv->counter.ptr};
    if(!e) e = launch_serve(L, srv->grid, ctx->own_stream);
    if(!e) e = load_profiles_kernel();
    if(!e) e = cudaStreamSynchronize(ctx->own_stream);
    if(e) return cuda_error(ctx, e, "serving warm-up");
    return MSA_OK;
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
        if(!rc) rc = msa_create(cfg->device, &srv->adm);
        if(!rc) rc = msa_create(cfg->device, &srv->ori);
        if(!rc) {
            cudaMemPoolProps props{};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = cfg->device;
            if(cudaMemPoolCreate(&srv->pool, &props) != cudaSuccess) {
                cudaGetLastError();
                srv->pool = nullptr;
                rc = MSA_ERR_CUDA;
            } else {
                // Keep released memory in the pool for the next jobs, and never
                // let an allocation on one stream wait for another stream's work.
                uint64_t keep = ~0ull;
                int no = 0;
                cudaMemPoolSetAttribute(srv->pool, cudaMemPoolAttrReleaseThreshold, &keep);
                cudaMemPoolSetAttribute(srv->pool, cudaMemPoolReuseAllowInternalDependencies, &no);
                srv->adm->pool = srv->pool;
                srv->ori->pool = srv->pool;
                int least = 0, greatest = 0;
                cudaDeviceGetStreamPriorityRange(&least, &greatest);
                if(cudaStreamCreateWithPriority(&srv->adm_stream, cudaStreamNonBlocking, greatest) == cudaSuccess)
                    srv->adm->stream = srv->adm_stream;
                else
                    cudaGetLastError();
            }
        }
        if(rc) {
            if(srv->ori) msa_destroy(srv->ori);
            if(srv->adm) msa_destroy(srv->adm);
            if(srv->ctx) msa_destroy(srv->ctx);
            delete srv;
            return rc;
        }
        size_t free_b = 0, total_b = 0;
        cudaSetDevice(cfg->device);
        if(cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) { cudaGetLastError(); free_b = 0; }
        srv->budget = cfg->hbm_budget_bytes ? cfg->hbm_budget_bytes : (uint64_t) (0.8 * (double) free_b);
        srv->max_jobs = cfg->max_jobs ? cfg->max_jobs : 64;
        srv->quantum = cfg->quantum_mcells;
        srv->window_ms = cfg->batch_window_us / 1000.0;
        srv->age_ms = cfg->age_weight_us / 1000.0;
        rc = warm_server(srv);
        if(rc) {
            srv->bound.release();
            srv->bound2.release();
            srv->tasks.release();
            srv->tasks2.release();
            srv->views.release();
            srv->views2.release();
            srv->counter.release();
            srv->counter2.release();
            msa_destroy(srv->ori);
            msa_destroy(srv->adm);
            if(srv->adm_stream) cudaStreamDestroy(srv->adm_stream);
            msa_destroy(srv->ctx);
            if(srv->pool) cudaMemPoolDestroy(srv->pool);
            delete srv;
            return rc;
        }
        srv->worker = std::thread(worker_loop, srv);
        {
            std::unique_lock<std::mutex> lk(srv->mu);
            srv->cv_done.wait(lk, [srv] { return srv->worker_ready; });
        }
        srv->t0 = now_ms();
        srv->orienter = std::thread(orientation_loop, srv);
        srv->admitter = std::thread(admission_loop, srv);
        *out = srv;
        return MSA_OK;
    } catch(...) {
        if(srv) {
            {
                std::lock_guard<std::mutex> lk(srv->mu);
                srv->stop = true;
            }
            srv->cv_work.notify_all();
            srv->cv_launch.notify_all();
            srv->cv_oriented.notify_all();
            if(srv->worker.joinable()) srv->worker.join();
            if(srv->admitter.joinable()) srv->admitter.join();
            if(srv->orienter.joinable()) srv->orienter.join();
            if(srv->ori) msa_destroy(srv->ori);
            if(srv->adm) msa_destroy(srv->adm);
            if(srv->adm_stream) cudaStreamDestroy(srv->adm_stream);
            if(srv->ctx) msa_destroy(srv->ctx);
            if(srv->pool) cudaMemPoolDestroy(srv->pool);
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
        if(srv->window_ms > 0) j->window = (uint64_t) std::ceil((j->t_submit - srv->t0) / srv->window_ms);
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
        srv->cv_launch.notify_all();
        srv->cv_oriented.notify_all();
    }
    if(srv->admitter.joinable()) srv->admitter.join();
    if(srv->orienter.joinable()) srv->orienter.join();
    if(srv->worker.joinable()) srv->worker.join();
    cudaSetDevice(srv->ctx->device);
    {
        // Fail what is still queued or admitted.
        std::lock_guard<std::mutex> lk(srv->mu);
        for(Job *j : srv->pending) { j->status = MSA_ERR_QUEUE; j->done = true; }
        srv->pending.clear();
        for(Job *j : srv->oriented) { j->status = MSA_ERR_QUEUE; j->done = true; }
        srv->oriented.clear();
        for(Job *j : srv->admitted) { release_job_device(j, srv->adm->stream); j->status = MSA_ERR_QUEUE; j->done = true; }
        srv->admitted.clear();
        srv->cv_done.notify_all();
        for(auto &kv : srv->jobs) delete kv.second;
        srv->jobs.clear();
    }
    cudaStreamSynchronize(srv->adm->stream);
    cudaStreamSynchronize(srv->ori->stream);
    srv->bound.release();
    srv->bound2.release();
    srv->tasks.release();
    srv->views.release();
    srv->counter.release();
    srv->tasks2.release();
    srv->views2.release();
    srv->counter2.release();
    msa_destroy(srv->ori);
    msa_destroy(srv->adm);
    if(srv->adm_stream) cudaStreamDestroy(srv->adm_stream);
    msa_destroy(srv->ctx);
    if(srv->pool) cudaMemPoolDestroy(srv->pool);
    delete srv;
    return MSA_OK;
}

}  // extern "C"
