// Internal declarations shared by the host runtime and the CUDA kernels of
// libmsa_b200.so. Nothing here crosses the C ABI.
#pragma once

#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>
#include <map>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/msa_b200.h"

namespace msa {

// Profile rows: encoder units 0..25 (24 = END never scored, 25 = GAP).
constexpr int kAlpha = 26;
// Profile rows are padded to a multiple of the tallest strip (32 lanes x 32 rows).
constexpr int kProfPad = 1024;
// Every sequence's units are padded with END so 16-byte loads past the end stay in bounds.
constexpr int kUnitPad = 64;

inline uint64_t round_up(uint64_t x, uint64_t m) { return (x + m - 1) / m * m; }

// Built-in tables in storage order (tables.inc).
struct BuiltinTable {
    const char *name;
    int32_t penalty;
    int8_t score[25 * 25];
};
const BuiltinTable *builtin_tables(int *count);

// Extended 26x26 table: entry [x][y] is what the reference reads for units x, y
// when it indexes `(*m_contents)[x][y]` on its contiguous table storage.
// valid[x*26+y] = 0 where that read would fall outside the storage.
struct ExtTable {
    int8_t score[kAlpha * kAlpha];
    uint8_t valid[kAlpha * kAlpha];
    int32_t penalty;
    int32_t max_abs;   // max |score| over valid entries (END row/column excluded)
    int32_t max_pos;   // largest score
    int32_t max_neg;   // largest magnitude of a negative score
    int32_t letter_pos;   // largest score among letter units (0..23), the only
    int32_t letter_neg;   // units of clean sequences; and its largest negative magnitude
};
int make_ext_table(const msa_table *t, ExtTable *out, std::string *err);

// Device-resident sequence store.
struct SeqStore {
    uint32_t n = 0;
    uint64_t serial = 0;            // unique per upload (plans are keyed by it)
    std::vector<uint64_t> len;      // given length (units)
    std::vector<uint32_t> eff;      // index of first END unit within the padded length
    std::vector<uint32_t> plen;     // 3 * ceil(len / 3)
    std::vector<uint8_t> dirty;     // END units not forming a suffix, or eff == 0
    std::vector<uint8_t> has_gap;   // a GAP unit within the padded length
    std::vector<uint64_t> off;      // byte offset of the units in d_units
    uint8_t *d_units = nullptr;
    uint64_t units_bytes = 0;
    uint64_t *d_off = nullptr;
    uint32_t *d_eff = nullptr;
    uint32_t *d_plen = nullptr;
    bool any_gap = false;
    // Clean sequences sorted by eff descending (ties: original index ascending).
    std::vector<uint32_t> clean_sorted;
    uint32_t *d_clean_sorted = nullptr;
    // Profile geometry per sequence (original index): Lp = round_up(max(eff,1), kProfPad).
    std::vector<uint64_t> prof_off;
    std::vector<uint32_t> prof_lp;
    uint64_t prof_bytes = 0;
    uint64_t *d_prof_off = nullptr;
    uint32_t *d_prof_lp = nullptr;
    std::vector<std::string> names;   // record descriptions (msa_seqs_load_fasta)
    // Device buffers came from the context's memory pool in stream order; they
    // are returned in stream order on free_stream.
    bool pooled = false;
    cudaStream_t free_stream = nullptr;
};

// Growable device scratch buffer owned by a context.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t need);
    void release();
};

struct GraphCache;

}  // namespace msa

struct msa_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    uint64_t launches = 0;
    std::map<uint64_t, msa::SeqStore *> stores;
    uint64_t next_handle = 1;
    int num_sms = 0;
    int cc_major = 0, cc_minor = 0;
    msa::DevBuf prof, bound, tasks, counters, out_tmp, pairs, nj_buf;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    msa_nw_stats last{};
    msa_nj_stats nj_last{};
    msa::GraphCache *graphs = nullptr;
    // When set, sequence stores are allocated from this pool on `stream`
    // (no device-wide synchronisation on allocation or release).
    cudaMemPool_t pool = nullptr;
    int tile_r = 0, tile_w = 0;   // persistent-kernel tile override (0 = autotuned)
    int nw_variant = 0;           // msa_nw_set_variant flags (0 = the committed kernel)
    uint32_t nw_chunk = 0;        // column groups per single-strip task (0 = autotuned)
    // msa_nj_set_clusters: clusters of the NJ launch (0 = automatic, 1 = one),
    // OTU count above which helpers scan (0 = default), wait limit between
    // clusters in microseconds (0 = default), and the stalled-publication test hook.
    int nj_clusters = 0;
    uint32_t nj_helper_c = 0, nj_wait_us = 0;
    int nj_stall = 0;
};

namespace msa {

// Kernel launchers (nw_kernels.cu). All launch on ctx->stream and count launches.
struct NwPlan;
// Scores the pairs of part `part` of `nparts` (split_job) into d_out; the
// other entries of d_out are not written. part 0 of 1 is the whole job.
int nw_run(msa_ctx *ctx, SeqStore *st, const ExtTable &tbl, int mode, int32_t *d_out, uint32_t part = 0,
           uint32_t nparts = 1);

// Host-side sequence scan (the rules of a store upload): index of the first
// END unit within the padded length, "dirty" (END units not forming a
// suffix, empty, or a GAP unit) and GAP presence.
void scan_units(const uint8_t *src, uint64_t len, uint32_t plen, uint32_t *eff, uint8_t *dirty, uint8_t *gap);
// Clean sequences sorted by eff descending (ties: index ascending).
void sort_clean(const std::vector<uint32_t> &eff, const std::vector<uint8_t> &dirty, std::vector<uint32_t> &out);
// Pairs with at least one dirty sequence, row-major, each as (rows, columns)
// in the reference's orientation.
void list_generic_pairs(const std::vector<uint8_t> &dirty, const std::vector<uint64_t> &len,
                        std::vector<uint32_t> &gpairs);
// A job cut into parts of about equal DP cells: rows pairs [k[p], k[p+1]) of
// the clean sorted order and generic pairs [g[p], g[p+1]).
struct JobSplit {
    std::vector<uint32_t> k;
    std::vector<uint64_t> g;
    std::vector<unsigned __int128> clean_cells;   // cumulative cells of rows pairs
};
JobSplit split_job(const std::vector<uint32_t> &eff, const std::vector<uint32_t> &plen,
                   const std::vector<uint32_t> &clean_sorted, const std::vector<uint32_t> &gpairs, uint32_t parts);
bool table_is_symmetric(const ExtTable &t);

// Bytes of padding before the first sequence in a store's unit buffer.
constexpr int kUnitFront = 64;
int nj_run(msa_ctx *ctx, const void *tri, int kind, uint32_t n, int order, msa_otu *out);

void release_graphs(msa_ctx *ctx);
int build_store(msa_ctx *ctx, const uint8_t *units, const uint64_t *offs, const uint64_t *lens, uint32_t n,
                SeqStore **out);
void destroy_store(SeqStore *st);
// Releases a pooled store's device memory in stream order on `s`.
void destroy_store_async(SeqStore *st, cudaStream_t s);
// Tile shape of the batched kernels for a store (committed autotuner table).
struct Tiles { int R, W; };
Tiles pick_tiles_for(const SeqStore *st);
// Score profiles of every sequence of a store into d_prof (st->prof_bytes).
cudaError_t launch_profiles(const SeqStore *st, const int8_t *d_ext, int8_t *d_prof, cudaStream_t s);
// 16-bit flag and column-group count of each rows pair (sorted 2k, 2k+1).
void plan_rows_pairs(const SeqStore *st, const ExtTable &tbl, Tiles tiles, std::vector<uint8_t> &narrow,
                     std::vector<uint32_t> &groups);
// One merged launch of the serving kernel (tiles 32 x 8) over `ntasks` tasks.
struct ServeLaunch {
    const void *jobs;        // JobView[slots], device
    const void *tasks;       // uint4[ntasks] (slot, rows pair, group, 0), device
    uint64_t ntasks;
    uint32_t *bound;
    uint64_t bound_stride;
    unsigned long long *counter;
};
int serve_grid(msa_ctx *ctx, uint64_t *grid);
cudaError_t load_profiles_kernel();   // loads the profile kernel's code on the current device
cudaError_t launch_serve(const ServeLaunch &l, uint64_t grid, cudaStream_t s);
size_t job_view_bytes();
void fill_job_view(void *dst, const SeqStore *st, const int8_t *d_prof, const uint8_t *d_narrow, int32_t *d_out,
                   int32_t g);
void drop_plans_for_store(msa_ctx *ctx, uint64_t serial);
int set_error(msa_ctx *ctx, int status, const std::string &msg);
int cuda_error(msa_ctx *ctx, cudaError_t e, const char *what);

}  // namespace msa

#define MSA_CUDA_TRY(ctx, call)                                             \
    do {                                                                    \
        cudaError_t _e = (call);                                            \
        if(_e != cudaSuccess) return msa::cuda_error((ctx), _e, #call);     \
    } while(0)
