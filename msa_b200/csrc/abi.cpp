// C ABI of libmsa_b200.so: contexts, the device-resident sequence store and
// the all-pairs NW / NJ entry points. Every entry point catches everything
// and returns a status; nothing throws across the boundary.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <new>
#include <numeric>
#include <string>

#include "msa_internal.hpp"

namespace msa {

cudaError_t DevBuf::ensure(size_t need)
{
    if(need <= bytes && ptr) return cudaSuccess;
    if(ptr) { cudaFree(ptr); ptr = nullptr; bytes = 0; }
    size_t want = std::max<size_t>(need, 256);
    cudaError_t e = cudaMalloc(&ptr, want);
    if(e != cudaSuccess) { ptr = nullptr; bytes = 0; cudaGetLastError(); return e; }
    bytes = want;
    return cudaSuccess;
}

void DevBuf::release()
{
    if(ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

int set_error(msa_ctx *ctx, int status, const std::string &msg)
{
    if(ctx) ctx->err = msg;
    return status;
}

int cuda_error(msa_ctx *ctx, cudaError_t e, const char *what)
{
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    return set_error(ctx, e == cudaErrorMemoryAllocation ? MSA_ERR_NOMEM : MSA_ERR_CUDA, m);
}

static void free_store(SeqStore *st)
{
    if(!st) return;
    void *bufs[] = {st->d_units, st->d_off, st->d_eff, st->d_plen, st->d_clean_sorted, st->d_prof_off, st->d_prof_lp};
    for(void *p : bufs) {
        if(!p) continue;
        if(st->pooled) cudaFreeAsync(p, st->free_stream);
        else cudaFree(p);
    }
    delete st;
}

}  // namespace msa

using namespace msa;

extern "C" {

int msa_create(int device, msa_ctx **out)
{
    if(!out) return MSA_ERR_INVALID;
    *out = nullptr;
    try {
        int count = 0;
        if(cudaGetDeviceCount(&count) != cudaSuccess || count == 0) { cudaGetLastError(); return MSA_ERR_NO_DEVICE; }
        if(device < 0 || device >= count) return MSA_ERR_INVALID;
        if(cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return MSA_ERR_CUDA; }
        cudaDeviceProp prop;
        if(cudaGetDeviceProperties(&prop, device) != cudaSuccess) { cudaGetLastError(); return MSA_ERR_CUDA; }
        if(prop.major < 10) return MSA_ERR_NO_DEVICE;   // built for sm_100a only
        auto *ctx = new msa_ctx;
        ctx->device = device;
        ctx->num_sms = prop.multiProcessorCount;
        ctx->cc_major = prop.major;
        ctx->cc_minor = prop.minor;
        if(cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            delete ctx;
            return MSA_ERR_CUDA;
        }
        ctx->stream = ctx->own_stream;
        for(auto &e : ctx->ev) cudaEventCreate(&e);
        *out = ctx;
        return MSA_OK;
    } catch(const std::bad_alloc &) {
        return MSA_ERR_NOMEM;
    } catch(...) {
        return MSA_ERR_CUDA;
    }
}

void msa_destroy(msa_ctx *ctx)
{
    if(!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    release_graphs(ctx);
    for(auto &kv : ctx->stores) free_store(kv.second);
    ctx->prof.release();
    ctx->bound.release();
    ctx->tasks.release();
    ctx->counters.release();
    ctx->out_tmp.release();
    ctx->pairs.release();
    ctx->nj_buf.release();
    for(auto &e : ctx->ev) if(e) cudaEventDestroy(e);
    if(ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
}

const char *msa_last_error(const msa_ctx *ctx) { return ctx ? ctx->err.c_str() : ""; }

int msa_set_stream(msa_ctx *ctx, void *stream)
{
    if(!ctx) return MSA_ERR_INVALID;
    ctx->stream = stream ? (cudaStream_t) stream : ctx->own_stream;
    return MSA_OK;
}

void *msa_get_stream(msa_ctx *ctx) { return ctx ? (void *) ctx->stream : nullptr; }

uint64_t msa_launch_count(const msa_ctx *ctx) { return ctx ? ctx->launches : 0; }

}  // extern "C"

namespace msa {

// Builds a device-resident store (the work of msa_seqs_upload without the
// handle). On failure nothing is left allocated.
int build_store(msa_ctx *ctx, const uint8_t *units, const uint64_t *offs, const uint64_t *lens, uint32_t n,
                SeqStore **out)
{
    if(!ctx || !out || (n && (!offs || !lens))) return MSA_ERR_INVALID;
    SeqStore *st = nullptr;
    try {
        cudaSetDevice(ctx->device);
        st = new SeqStore;
        st->n = n;
        st->len.resize(n);
        st->eff.resize(n);
        st->plen.resize(n);
        st->dirty.resize(n);
        st->has_gap.resize(n);
        st->off.resize(n);
        uint64_t total = kUnitFront;   // lanes may read a few residues before a sequence
        for(uint32_t i = 0; i < n; ++i) {
            const uint64_t L = lens[i];
            if(L >= (1ull << 30)) { free_store(st); return set_error(ctx, MSA_ERR_TOO_LARGE, "sequence longer than 2^30 units"); }
            if(L && !units) { free_store(st); return MSA_ERR_INVALID; }
            st->len[i] = L;
            st->plen[i] = (uint32_t) ((L + 2) / 3 * 3);
            st->off[i] = total;
            total += round_up(st->plen[i] + kUnitPad, 16);
        }
        st->units_bytes = total + kUnitPad;
        std::vector<uint8_t> host(st->units_bytes, (uint8_t) MSA_UNIT_END);
        for(uint32_t i = 0; i < n; ++i) {
            const uint8_t *src = units + offs[i];
            uint8_t *dst = host.data() + st->off[i];
            for(uint64_t k = 0; k < st->len[i]; ++k) {
                const uint8_t u = src[k];
                if(u > MSA_UNIT_GAP) { free_store(st); return set_error(ctx, MSA_ERR_INVALID, "unit code above 25"); }
                dst[k] = u;
            }
            scan_units(src, st->len[i], st->plen[i], &st->eff[i], &st->dirty[i], &st->has_gap[i]);
            st->any_gap |= st->has_gap[i] != 0;
        }
        // Clean sequences sorted by effective length, longest first.
        sort_clean(st->eff, st->dirty, st->clean_sorted);
        // Profile geometry.
        st->prof_off.resize(n);
        st->prof_lp.resize(n);
        uint64_t poff = 0;
        for(uint32_t i = 0; i < n; ++i) {
            st->prof_lp[i] = (uint32_t) round_up(std::max<uint32_t>(st->eff[i], 1), kProfPad);
            st->prof_off[i] = poff;
            poff += (uint64_t) kAlpha * st->prof_lp[i];
        }
        st->prof_bytes = poff;

        st->pooled = ctx->pool != nullptr;
        st->free_stream = ctx->stream;
        auto dmalloc = [&](void **p, size_t b) {
            return st->pooled ? cudaMallocFromPoolAsync(p, std::max<size_t>(b, 16), ctx->pool, ctx->stream)
                              : cudaMalloc(p, std::max<size_t>(b, 16));
        };
        cudaError_t e = cudaSuccess;
        if(!e) e = dmalloc((void **) &st->d_units, st->units_bytes);
        if(!e) e = dmalloc((void **) &st->d_off, n * sizeof(uint64_t));
        if(!e) e = dmalloc((void **) &st->d_eff, n * sizeof(uint32_t));
        if(!e) e = dmalloc((void **) &st->d_plen, n * sizeof(uint32_t));
        if(!e) e = dmalloc((void **) &st->d_clean_sorted, st->clean_sorted.size() * sizeof(uint32_t));
        if(!e) e = dmalloc((void **) &st->d_prof_off, n * sizeof(uint64_t));
        if(!e) e = dmalloc((void **) &st->d_prof_lp, n * sizeof(uint32_t));
        cudaStream_t s = ctx->stream;
        if(!e) e = cudaMemcpyAsync(st->d_units, host.data(), st->units_bytes, cudaMemcpyHostToDevice, s);
        if(!e && n) e = cudaMemcpyAsync(st->d_off, st->off.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, s);
        if(!e && n) e = cudaMemcpyAsync(st->d_eff, st->eff.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, s);
        if(!e && n) e = cudaMemcpyAsync(st->d_plen, st->plen.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, s);
        if(!e && !st->clean_sorted.empty())
            e = cudaMemcpyAsync(st->d_clean_sorted, st->clean_sorted.data(), st->clean_sorted.size() * sizeof(uint32_t),
                                cudaMemcpyHostToDevice, s);
        if(!e && n) e = cudaMemcpyAsync(st->d_prof_off, st->prof_off.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, s);
        if(!e && n) e = cudaMemcpyAsync(st->d_prof_lp, st->prof_lp.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, s);
        if(!e) e = cudaStreamSynchronize(s);   // host staging buffer goes out of scope
        if(e) { free_store(st); return cuda_error(ctx, e, "sequence upload"); }
        static std::atomic<uint64_t> serials{1};
        st->serial = serials++;
        *out = st;
        return MSA_OK;
    } catch(const std::bad_alloc &) {
        free_store(st);
        return set_error(ctx, MSA_ERR_NOMEM, "host allocation failed");
    } catch(...) {
        free_store(st);
        return set_error(ctx, MSA_ERR_CUDA, "unexpected failure building a sequence store");
    }
}

void destroy_store(SeqStore *st) { free_store(st); }

void destroy_store_async(SeqStore *st, cudaStream_t s)
{
    if(st && st->pooled) st->free_stream = s;
    free_store(st);
}

}  // namespace msa

extern "C" int msa_seqs_upload(msa_ctx *ctx, const uint8_t *units, const uint64_t *offs, const uint64_t *lens,
                               uint32_t n, msa_seqs *out)
{
    if(!ctx || !out) return MSA_ERR_INVALID;
    SeqStore *st = nullptr;
    const int rc = msa::build_store(ctx, units, offs, lens, n, &st);
    if(rc) return rc;
    try {
        const uint64_t h = ctx->next_handle++;
        ctx->stores[h] = st;
        *out = h;
        return MSA_OK;
    } catch(...) {
        free_store(st);
        return set_error(ctx, MSA_ERR_NOMEM, "host allocation failed");
    }
}

extern "C" {

int msa_seqs_release(msa_ctx *ctx, msa_seqs seqs)
{
    if(!ctx) return MSA_ERR_INVALID;
    auto it = ctx->stores.find(seqs);
    if(it == ctx->stores.end()) return MSA_ERR_HANDLE;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    drop_plans_for_store(ctx, it->second->serial);
    free_store(it->second);
    ctx->stores.erase(it);
    return MSA_OK;
}

int64_t msa_seqs_count(msa_ctx *ctx, msa_seqs seqs)
{
    if(!ctx) return -1;
    auto it = ctx->stores.find(seqs);
    return it == ctx->stores.end() ? -1 : (int64_t) it->second->n;
}

}  // extern "C"

namespace msa {

bool table_is_symmetric(const ExtTable &t)
{
    for(int x = 0; x < 25; ++x)
        for(int y = 0; y < 25; ++y)
            if(t.score[x * kAlpha + y] != t.score[y * kAlpha + x]) return false;
    return true;
}

static int all_pairs(msa_ctx *ctx, msa_seqs seqs, const msa_table *table, int mode, uint32_t part, uint32_t nparts,
                     int32_t *out, int out_on_device)
{
    if(!ctx || !table || nparts == 0 || part >= nparts) return MSA_ERR_INVALID;
    try {
        auto it = ctx->stores.find(seqs);
        if(it == ctx->stores.end()) return set_error(ctx, MSA_ERR_HANDLE, "unknown sequence store");
        SeqStore *st = it->second;
        if(mode != MSA_NW_AUTO && mode != MSA_NW_PLAIN && mode != MSA_NW_PERSISTENT)
            return set_error(ctx, MSA_ERR_UNKNOWN_ALGORITHM, "unknown NW mode");
        if(mode == MSA_NW_AUTO) mode = MSA_NW_PERSISTENT;
        cudaSetDevice(ctx->device);
        ExtTable ext;
        std::string err;
        int rc = make_ext_table(table, &ext, &err);
        if(rc) return set_error(ctx, rc, err);
        // A GAP unit is scored through the reference's flat table storage; where
        // that read leaves the storage the reference is undefined.
        if(st->any_gap) {
            for(int x = 0; x < kAlpha; ++x)
                for(int y = 0; y < kAlpha; ++y)
                    if((x == MSA_UNIT_GAP || y == MSA_UNIT_GAP) && x != MSA_UNIT_END && y != MSA_UNIT_END &&
                       !ext.valid[x * kAlpha + y])
                        return set_error(ctx, MSA_ERR_UNDEFINED,
                                         "GAP unit with this table reads past the reference's table storage");
        }
        // Exact parity with float scores needs |score| < 2^24; int32 needs < 2^31.
        uint64_t maxlen = 0;
        for(uint32_t i = 0; i < st->n; ++i) maxlen = std::max<uint64_t>(maxlen, st->plen[i]);
        const int64_t vb = (int64_t) (2 * maxlen + 2048 + 2) * std::max<int64_t>(ext.max_abs, ext.penalty);
        if(vb >= (1ll << 30)) return set_error(ctx, MSA_ERR_TOO_LARGE, "scores could exceed the int32 range");
        const uint64_t npairs = (uint64_t) st->n * (st->n ? st->n - 1 : 0) / 2;
        if(npairs && !out) return MSA_ERR_INVALID;
        // Tables that are not symmetric make the score depend on orientation:
        // route every pair through the reference-orientation path for this
        // call. The store's own plan comes back on every exit, exceptions
        // included.
        struct Reorient {
            SeqStore *st;
            bool active;
            std::vector<uint8_t> dirty;
            std::vector<uint32_t> sorted;
            Reorient(SeqStore *s, bool on) : st(s), active(on)
            {
                if(!active) return;
                dirty = st->dirty;
                sorted = st->clean_sorted;
                std::fill(st->dirty.begin(), st->dirty.end(), 1);
                st->clean_sorted.clear();
            }
            ~Reorient()
            {
                if(!active) return;
                st->dirty.swap(dirty);
                st->clean_sorted.swap(sorted);
            }
        } reorient(st, !table_is_symmetric(ext));
        int32_t *d_out = out;
        if(!out_on_device && npairs) {
            cudaError_t e = ctx->out_tmp.ensure(npairs * sizeof(int32_t));
            if(e) return cuda_error(ctx, e, "output buffer");
            d_out = (int32_t *) ctx->out_tmp.ptr;
        }
        rc = nw_run(ctx, st, ext, mode, d_out, part, nparts);
        std::vector<uint32_t> owner;
        if(!out_on_device && npairs && nparts > 1 && !rc) {
            // Host output of one part: only that part's entries are written.
            owner.resize(npairs);
            std::vector<uint32_t> gpairs;
            list_generic_pairs(st->dirty, st->len, gpairs);
            const JobSplit s = split_job(st->eff, st->plen, st->clean_sorted, gpairs, nparts);
            std::fill(owner.begin(), owner.end(), nparts);
            auto tri = [](uint64_t i, uint64_t j) { return i > j ? i * (i - 1) / 2 + j : j * (j - 1) / 2 + i; };
            const auto &cs = st->clean_sorted;
            for(uint32_t k = s.k[part]; k < s.k[part + 1]; ++k)
                for(uint32_t a = 2 * k; a < std::min<uint32_t>(2 * k + 2, (uint32_t) cs.size()); ++a)
                    for(uint32_t b = a + 1; b < (uint32_t) cs.size(); ++b) owner[tri(cs[a], cs[b])] = part;
            for(uint64_t q = s.g[part]; q < s.g[part + 1]; ++q) owner[tri(gpairs[2 * q], gpairs[2 * q + 1])] = part;
        }
        if(rc) return rc;
        if(!out_on_device && npairs) {
            if(nparts == 1) {
                cudaError_t e = cudaMemcpyAsync(out, d_out, npairs * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream);
                if(!e) e = cudaStreamSynchronize(ctx->stream);
                if(e) return cuda_error(ctx, e, "copy scores to host");
            } else {
                std::vector<int32_t> all(npairs);
                cudaError_t e = cudaMemcpyAsync(all.data(), d_out, npairs * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                                ctx->stream);
                if(!e) e = cudaStreamSynchronize(ctx->stream);
                if(e) return cuda_error(ctx, e, "copy scores to host");
                for(uint64_t q = 0; q < npairs; ++q)
                    if(owner[q] == part) out[q] = all[q];
            }
        }
        return MSA_OK;
    } catch(const std::bad_alloc &) {
        return set_error(ctx, MSA_ERR_NOMEM, "host allocation failed");
    } catch(...) {
        return set_error(ctx, MSA_ERR_CUDA, "unexpected failure in msa_nw_all_pairs");
    }
}

}  // namespace msa

extern "C" {

int msa_nw_all_pairs(msa_ctx *ctx, msa_seqs seqs, const msa_table *table, int mode, int32_t *out,
                     int out_on_device)
{
    return msa::all_pairs(ctx, seqs, table, mode, 0, 1, out, out_on_device);
}

int msa_nw_all_pairs_part(msa_ctx *ctx, msa_seqs seqs, const msa_table *table, int mode, uint32_t part,
                          uint32_t nparts, int32_t *out, int out_on_device)
{
    return msa::all_pairs(ctx, seqs, table, mode, part, nparts, out, out_on_device);
}

int msa_nw_set_variant(msa_ctx *ctx, int flags, uint32_t groups_per_task)
{
    if(!ctx) return MSA_ERR_INVALID;
    if(flags & ~(MSA_NW_VARIANT_INT32 | MSA_NW_VARIANT_NO_PACKED)) return MSA_ERR_INVALID;
    if(groups_per_task > 64) return MSA_ERR_INVALID;
    ctx->nw_variant = flags;
    ctx->nw_chunk = groups_per_task;
    return MSA_OK;
}

int msa_nw_set_tiles(msa_ctx *ctx, int rows_per_lane, int warps_per_cta)
{
    if(!ctx) return MSA_ERR_INVALID;
    if(rows_per_lane == 0 && warps_per_cta == 0) { ctx->tile_r = ctx->tile_w = 0; return MSA_OK; }
    if((rows_per_lane != 16 && rows_per_lane != 32) || (warps_per_cta != 4 && warps_per_cta != 8))
        return MSA_ERR_INVALID;
    ctx->tile_r = rows_per_lane;
    ctx->tile_w = warps_per_cta;
    return MSA_OK;
}

int msa_nw_last_stats(const msa_ctx *ctx, msa_nw_stats *out)
{
    if(!ctx || !out) return MSA_ERR_INVALID;
    *out = ctx->last;
    return MSA_OK;
}

int msa_nj_set_clusters(msa_ctx *ctx, int clusters, uint32_t helper_min_count, uint32_t wait_limit_us,
                        int stall_publication)
{
    if(!ctx || clusters < 0 || clusters > 9) return MSA_ERR_INVALID;
    ctx->nj_clusters = clusters;
    ctx->nj_helper_c = helper_min_count;
    ctx->nj_wait_us = wait_limit_us;
    ctx->nj_stall = stall_publication ? 1 : 0;
    return MSA_OK;
}

int msa_nj_last_stats(const msa_ctx *ctx, msa_nj_stats *out)
{
    if(!ctx || !out) return MSA_ERR_INVALID;
    *out = ctx->nj_last;
    return MSA_OK;
}

int msa_nj(msa_ctx *ctx, const void *tri, int tri_kind, uint32_t n, msa_otu *out_nodes)
{
    return msa_nj_order(ctx, tri, tri_kind, n, MSA_NJ_SYMMETRIC, out_nodes);
}

int msa_nj_order(msa_ctx *ctx, const void *tri, int tri_kind, uint32_t n, int order, msa_otu *out_nodes)
{
    if(!ctx) return MSA_ERR_INVALID;
    if(order != MSA_NJ_SYMMETRIC && order != MSA_NJ_LINEAR) return MSA_ERR_INVALID;
    if(n < 2) return MSA_OK;
    if(!tri || !out_nodes) return MSA_ERR_INVALID;
    if(tri_kind < MSA_TRI_F32_HOST || tri_kind > MSA_TRI_I32_DEVICE) return MSA_ERR_INVALID;
    try {
        cudaSetDevice(ctx->device);
        return nj_run(ctx, tri, tri_kind, n, order, out_nodes);
    } catch(const std::bad_alloc &) {
        return set_error(ctx, MSA_ERR_NOMEM, "host allocation failed");
    } catch(...) {
        return set_error(ctx, MSA_ERR_CUDA, "unexpected failure in msa_nj");
    }
}

}  // extern "C"
