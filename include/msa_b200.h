/*
 * msa_b200 — C ABI of the B200-native all-pairs Needleman-Wunsch and
 * neighbor-joining library (libmsa_b200.so).
 *
 * Plain pointers and sizes only. Every entry point returns an msa_status;
 * nothing throws across this boundary. A context owns one CUDA stream and
 * the device buffers it allocates; use one context per host thread.
 *
 * Each declaration names the reference interface it replaces (Museqa
 * v0.1.1, paths relative to the project root).
 */
#ifndef MSA_B200_H
#define MSA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */

typedef enum msa_status {
    MSA_OK = 0,
    MSA_ERR_INVALID = 1,            /* bad argument (null pointer, size, unit code) */
    MSA_ERR_CUDA = 2,               /* a CUDA runtime call failed; see msa_last_error */
    MSA_ERR_NOMEM = 3,              /* device or host allocation failed */
    MSA_ERR_UNKNOWN_TABLE = 4,      /* "unknown pairwise scoring table '%s'" (src/pairwise/table.cu:315-321) */
    MSA_ERR_UNKNOWN_ALGORITHM = 5,  /* "unknown pairwise/phylogeny algorithm '%s'" (src/pairwise/pairwise.cpp:298-303) */
    MSA_ERR_HANDLE = 6,             /* stale or foreign sequence-store handle */
    MSA_ERR_DEVICE_TIMEOUT = 7,     /* a bounded device-side wait gave up; the context stays usable */
    MSA_ERR_UNDEFINED = 8,          /* input whose result the reference leaves undefined (see msa_nw_all_pairs) */
    MSA_ERR_NO_DEVICE = 9,          /* no CUDA device, or the library was built without a usable kernel image */
    MSA_ERR_QUEUE = 10,             /* serving queue closed, full, or job id unknown */
    MSA_ERR_TOO_LARGE = 11          /* request exceeds a stated size limit */
} msa_status;

/* Message for a status code. */
const char *msa_strerror(int status);

/* ----------------------------------------------------------------- tables */

/* Number of scoring-table entries per side; rows and columns are encoder units. */
#define MSA_TABLE_SIDE 25

/*
 * A scoring table by value: scoring_table (src/pairwise/pairwise.cuh:124-182).
 * `score[x*25+y]` is the score of units x and y; `penalty` is the positive
 * linear gap penalty that is subtracted. `index` is the table's position in
 * the built-in storage order (default, blosum62, blosum45, blosum50,
 * blosum80, blosum90, pam250; src/pairwise/table.cu:41-262), or -1 for a
 * caller-made table.
 */
typedef struct msa_table {
    int32_t score[MSA_TABLE_SIDE * MSA_TABLE_SIDE];
    int32_t penalty;
    int32_t index;
} msa_table;

/* scoring_table::make(name) (src/pairwise/table.cu:315-321). */
int msa_table_make(const char *name, msa_table *out);
/* scoring_table::has(name) (src/pairwise/table.cu:305-308): 1 or 0. */
int msa_table_has(const char *name);
/* scoring_table::list() (src/pairwise/table.cu:327-330): names in the
 * reference's (sorted) order. Returns the count; fills up to `cap` names. */
int msa_table_list(const char **names, int cap);

/* ---------------------------------------------------------------- encoder */

/* Unit codes (src/encoder.hpp:42-48). */
#define MSA_UNIT_END 0x18
#define MSA_UNIT_GAP 0x19

/* encoder::encode(char) (src/encoder.cpp:46-57) over `len` characters into
 * one byte per unit. */
int msa_encode(const char *chars, uint64_t len, uint8_t *out_units);
/* encoder::decode(unit) (src/encoder.cpp:36-39, :62-66) into characters. */
int msa_decode(const uint8_t *units, uint64_t len, char *out_chars);
/* encoder::encode(const char*, size_t) (src/encoder.cpp:76-98): the
 * reference's packed form, 3 units per uint16 block, bit 0 = padded block.
 * Returns MSA_OK; ceil(len/3) blocks written. */
int msa_encode_blocks(const char *chars, uint64_t len, uint16_t *out_blocks);
/* Inverse of the packed form: 3*nblocks units. */
int msa_unpack_blocks(const uint16_t *blocks, uint64_t nblocks, uint8_t *out_units);

/* ---------------------------------------------------------------- context */

typedef struct msa_ctx msa_ctx;

/* Creates a context on `device` (the CLI's -d/--device, src/museqa.cpp:34). */
int msa_create(int device, msa_ctx **out);
void msa_destroy(msa_ctx *ctx);
/* Detail of the context's last failure (empty if none). */
const char *msa_last_error(const msa_ctx *ctx);
/* Makes the context launch on `stream` (a cudaStream_t; NULL = the context's
 * own stream). The caller keeps the stream alive while the context uses it. */
int msa_set_stream(msa_ctx *ctx, void *stream);
void *msa_get_stream(msa_ctx *ctx);
/* Number of this library's kernel launches issued by the context so far. */
uint64_t msa_launch_count(const msa_ctx *ctx);

/* ---------------------------------------------------------- sequence store */

typedef uint64_t msa_seqs;

/*
 * Uploads n sequences of encoder units into device memory: the device-resident
 * replacement of pairwise::database (src/pairwise/database.cuh:27-91,
 * src/pairwise/database.cu:24-72). Sequence k is units[offs[k] .. offs[k]+lens[k]).
 * Units past lens[k] up to the next multiple of 3 are END, as in the
 * reference's block padding (src/sequence.hpp:101-104). Unit codes must be
 * 0..25. The caller's arrays may be freed after the call returns.
 */
int msa_seqs_upload(msa_ctx *ctx, const uint8_t *units, const uint64_t *offs,
                    const uint64_t *lens, uint32_t n, msa_seqs *out);
int msa_seqs_release(msa_ctx *ctx, msa_seqs seqs);
/* Number of sequences in a store, or -1 for a bad handle. */
int64_t msa_seqs_count(msa_ctx *ctx, msa_seqs seqs);

/*
 * FASTA files straight into a device store: the reference's loader
 * (io::loader by extension, src/io/loader/database.cpp:31-52; parser::fasta,
 * src/io/loader/parser/fasta.cpp:26-70; encoder::encode, src/encoder.cpp:46-57)
 * in one pass per file, then one upload. Records keep the reference's rules:
 * contents are the lines after a '>' line up to the next '>' line or the first
 * empty line, '\r' stays (and encodes as END), only "fa"/"fasta" files are read.
 * *count receives the number of records; their descriptions stay with the store
 * (msa_seqs_description).
 */
int msa_seqs_load_fasta(msa_ctx *ctx, const char *const *files, uint32_t nfiles, msa_seqs *out, uint32_t *count);
/* Description of record `index` of a store made by msa_seqs_load_fasta, valid
 * until the store is released; NULL otherwise. */
const char *msa_seqs_description(msa_ctx *ctx, msa_seqs seqs, uint32_t index);
/* Host-only halves of the same loader: the record count and total units, then
 * the units (one byte each, unpadded), offsets and lengths, as msa_seqs_upload
 * takes them. */
int msa_fasta_count(const char *const *files, uint32_t nfiles, uint32_t *nseqs, uint64_t *nunits);
int msa_fasta_encode(const char *const *files, uint32_t nfiles, uint8_t *units, uint64_t *offs, uint64_t *lens);

/* ---------------------------------------------------------- all-pairs NW */

typedef enum msa_nw_mode {
    MSA_NW_AUTO = 0,        /* = MSA_NW_PERSISTENT */
    MSA_NW_PLAIN = 1,       /* one launch per length bucket, one pair per warp, int32 */
    MSA_NW_PERSISTENT = 2   /* one persistent work-stealing launch over cost-ordered tiles,
                               autotuned tile shapes, 16-bit lanes where provably exact,
                               replayed from a CUDA graph */
} msa_nw_mode;

/*
 * Scores every pair i > j of the store with global linear-gap
 * Needleman-Wunsch and writes out[i*(i-1)/2 + j] (int32): the scoring step of
 * needleman::sequential / needleman::hybrid
 * (src/pairwise/needleman/impl/sequential.cpp:29-122,
 * src/pairwise/needleman/impl/hybrid.cu:403-456) with the packed
 * lower-triangle layout of distance_matrix (src/pairwise/pairwise.cuh:53-117).
 * Scores equal the reference's float scores exactly (they are small integers);
 * the reference's treatment of END units inside a sequence (row truncation,
 * column skipping) is reproduced.
 *
 * `out` is host memory (out_on_device = 0) or device memory of this context's
 * device (out_on_device = 1). Returns MSA_ERR_UNDEFINED when a GAP unit (25)
 * would index past the reference's table storage (pam250 or a caller table),
 * which is undefined behaviour in the reference.
 */
int msa_nw_all_pairs(msa_ctx *ctx, msa_seqs seqs, const msa_table *table, int mode,
                     int32_t *out, int out_on_device);

/*
 * One part of an all-pairs job split over several devices. Replaces the
 * reference's MPI split of the pair list over ranks
 * (src/pairwise/needleman/needleman.cpp:31-52, utils::partition at
 * src/utils.hpp:176-183), which gives every rank the same number of pairs;
 * here the parts hold about equal DP cells. Scores exactly the pairs that
 * msa_nw_part_of_pairs assigns to `part` (0 <= part < nparts) and writes
 * only their entries of `out` (n(n-1)/2 int32 at i(i-1)/2+j); every other
 * entry keeps its value. Scores equal msa_nw_all_pairs's. Every device given
 * the same sequences, table, mode and nparts computes the same split, so
 * zero-filled outputs of all parts summed (or the parts written into one
 * buffer) give the whole matrix.
 */
int msa_nw_all_pairs_part(msa_ctx *ctx, msa_seqs seqs, const msa_table *table, int mode, uint32_t part,
                          uint32_t nparts, int32_t *out, int out_on_device);

/* Host-only: the part (0..nparts-1) that msa_nw_all_pairs_part assigns to
 * every pair, written at i(i-1)/2+j of `out_part` (n(n-1)/2 entries). Needs
 * no device. */
int msa_nw_part_of_pairs(const uint8_t *units, const uint64_t *offs, const uint64_t *lens, uint32_t n,
                         const msa_table *table, uint32_t nparts, uint32_t *out_part);

/* Tile shape of the persistent kernel: rows per lane (16 or 32) and warps per
 * CTA (4 or 8); 0, 0 restores the committed autotuned choice. No counterpart
 * in the reference (its one kernel shape is fixed, hybrid.cu:57). */
int msa_nw_set_tiles(msa_ctx *ctx, int rows_per_lane, int warps_per_cta);

/* Variants of the persistent kernel, for measuring what each of its parts
 * contributes (no counterpart in the reference, which has one kernel). Flags:
 * MSA_NW_VARIANT_INT32 runs every task in 32-bit lanes (one rows sequence at
 * a time); MSA_NW_VARIANT_NO_PACKED stages every profile row as 16-bit words,
 * with 32x8 tiles. groups_per_task (0 = the autotuned choice, at most 64) is
 * how many column groups a task of a rows pair that fits one strip sweeps
 * after one staging of that strip; 1 restages it for every group. Scores are
 * the same under every setting. Applies to later calls on the context. */
#define MSA_NW_VARIANT_INT32 1
#define MSA_NW_VARIANT_NO_PACKED 2
int msa_nw_set_variant(msa_ctx *ctx, int flags, uint32_t groups_per_task);

/* Timing breakdown of the context's last msa_nw_all_pairs call (device ms). */
typedef struct msa_nw_stats {
    double kernel_ms;       /* NW kernels only */
    double total_ms;        /* whole device-side call, profile build included */
    uint64_t cells;         /* sum over pairs of (effective rows x effective columns) */
    uint64_t pairs;
    uint32_t launches;      /* kernel launches issued by the call */
    uint32_t narrow_tasks;  /* tasks run on 16-bit lanes */
    uint32_t graph;         /* 1 if the call replayed a captured CUDA graph */
} msa_nw_stats;
int msa_nw_last_stats(const msa_ctx *ctx, msa_nw_stats *out);

/*
 * All-pairs NW that allocates nothing (no counterpart in the reference, which
 * always allocates per call). For callers that may not call cudaMalloc when
 * they score, e.g. a runtime that owns all device memory in its own pool, or
 * code that must avoid the device synchronisation an allocation can imply.
 * `units` (device) holds the sequences; `offs` and `lens` (host, n entries)
 * locate sequence k at units[offs[k] .. offs[k]+lens[k]); `out` (device) gets
 * n(n-1)/2 int32 scores at i(i-1)/2+j, equal to msa_nw_all_pairs (and, like
 * it, MSA_ERR_UNDEFINED when any sequence holds a GAP unit and the table's
 * GAP entries lie outside the reference's storage). Runs on `stream` (a
 * cudaStream_t, NULL = legacy default) of the current device; the call is
 * blocking: it synchronises `stream` and returns after the scores are written.
 * Scratch is one fixed 16 MiB device array inside this library, shared by all
 * calls on a device and keeping the last call's contents: calls that overlap
 * on the GPU race and must be serialised by the caller. The first call on a
 * device looks up that array's address, so make it before any stream capture.
 * Limits: n <= 65536 and sequences up to about one million units; larger
 * requests return MSA_ERR_TOO_LARGE. msa_noalloc_last_error() explains a
 * failure.
 */
int msa_nw_all_pairs_noalloc(const uint8_t *units, const uint64_t *offs, const uint64_t *lens,
                             uint32_t n, const msa_table *table, int32_t *out, void *stream);
const char *msa_noalloc_last_error(void);

/* ---------------------------------------------------------- neighbor-joining */

/* One node of the guide tree: otu + hierarchy
 * (src/phylogeny/phylogeny.cuh:171-180, src/hierarchy.hpp:46-47).
 * Undefined references are 0xFFFFFFFF. */
typedef struct msa_otu {
    uint32_t parent;
    uint32_t child[2];
    float distance;
    uint32_t level;
} msa_otu;

typedef enum msa_tri_kind {
    MSA_TRI_F32_HOST = 0,
    MSA_TRI_F32_DEVICE = 1,
    MSA_TRI_I32_HOST = 2,
    MSA_TRI_I32_DEVICE = 3
} msa_tri_kind;

/*
 * Neighbor-joining over the packed lower triangle `tri` (n(n-1)/2 values,
 * index i(i-1)/2+j; int32 kinds are converted to float exactly): the
 * replacement of njoining::sequential_symmetric / hybrid_symmetric
 * (src/phylogeny/njoining/impl/sequential.cpp:80-346,
 * src/phylogeny/njoining/impl/hybrid.cu:149-543). Writes 2n-1 nodes, leaves
 * 0..n-1, parents n..2n-2 in join order, root 2n-2. The joins, branch lengths
 * and levels equal the reference's sequential symmetric algorithm bit for bit.
 * n < 2 writes nothing (phylogeny returns an empty tree).
 */
int msa_nj(msa_ctx *ctx, const void *tri, int tri_kind, uint32_t n, msa_otu *out_nodes);

/* Removal order of a neighbor-joining run: the reference's two matrix
 * transforms (src/phylogeny/njoining/impl/sequential.cpp:189-224). After a
 * join of (x, y), SYMMETRIC swaps y with logical 0 and drops logical 0, so
 * every index moves down by one; LINEAR swaps y with the last logical OTU and
 * drops the last. The first-maximum tie-break scans in that order, so the two
 * give different trees (and always different branch-length bits). */
typedef enum msa_nj_order_kind {
    MSA_NJ_SYMMETRIC = 0,
    MSA_NJ_LINEAR = 1
} msa_nj_order_kind;

/*
 * msa_nj with the removal order chosen: MSA_NJ_SYMMETRIC is msa_nj;
 * MSA_NJ_LINEAR replaces njoining::sequential_linear / hybrid_linear
 * (src/phylogeny/njoining/impl/sequential.cpp:189-203, 356-358;
 * src/phylogeny/phylogeny.cpp:30,33,38,40) bit for bit. Other values give
 * MSA_ERR_INVALID.
 */
int msa_nj_order(msa_ctx *ctx, const void *tri, int tri_kind, uint32_t n, int order, msa_otu *out_nodes);

/* Timing of the context's last msa_nj call. The joins run on one cluster of
 * `cluster` CTAs; cycle counts are SM clock cycles by phase, for CTA 0 (scan,
 * wait for the candidates, join, wait until every CTA has read the joined
 * rows, writes) and for the CTA that folds each new node's row sum (the fold,
 * its scan of the new node's row, its wait for the candidates). */
typedef struct msa_nj_stats {
    double kernel_ms;
    double total_ms;            /* upload, matrix set-up, joins, download */
    uint32_t n;
    uint32_t cluster;
    uint64_t cycles_scan, cycles_wait, cycles_join, cycles_join_wait, cycles_write;
    uint64_t cycles_fold, cycles_fold_row, cycles_fold_wait;
    uint32_t helper_clusters;   /* clusters that scanned beside the joining one */
} msa_nj_stats;
int msa_nj_last_stats(const msa_ctx *ctx, msa_nj_stats *out);

/* How a neighbor-joining run spreads its search over the GPU (no counterpart
 * in the reference). One thread-block cluster makes every join; up to
 * `clusters` - 1 more clusters (0 = the default, which is none; 1 = none)
 * scan a share of the rows for each join while more than `helper_min_count`
 * OTUs remain (0 = the default, 1,400), exchanging candidates and row sums
 * through global memory; at most as many as are resident and 128 CTAs. Every
 * wait between clusters ends after `wait_limit_us` (0 = the default, 1 s);
 * a wait that runs out fails the call with MSA_ERR_DEVICE_TIMEOUT and leaves
 * the context usable. `stall_publication` != 0 is a test hook: the joining
 * cluster then never hands its row sums to the helpers, so their waits run
 * out. Trees are the same under every setting. Applies to later calls. */
int msa_nj_set_clusters(msa_ctx *ctx, int clusters, uint32_t helper_min_count, uint32_t wait_limit_us,
                        int stall_publication);

/* ---------------------------------------------------------------- serving */

typedef struct msa_server msa_server;

typedef struct msa_serve_config {
    int device;
    uint64_t hbm_budget_bytes;  /* 0 = 80 % of free device memory at start */
    uint32_t max_jobs;          /* admitted jobs at once; 0 = 64 */
    uint32_t quantum_mcells;    /* DP cells per merged launch, in millions; 0 = 40,000 */
    /* 0 (continuous admission): a job is admitted as soon as memory and a slot
     * allow, and every admitted job gets an equal share of each merged launch.
     * W > 0 (batch windows): a job is admitted at the first multiple of W
     * microseconds (from server start) after its submission; windows are
     * served in order, and the jobs of one window share the launches in
     * proportion to their remaining cells, so they finish together. The
     * next window's jobs are admitted while the previous one runs and fill
     * its last launches. */
    uint32_t batch_window_us;
    /* Under continuous admission only: 0 shares each merged launch equally
     * among the admitted jobs; A > 0 weights job i by 1 + age_i / A (age_i
     * the time since its submission, in microseconds), so a job that has
     * waited long, in practice a large one, takes a growing share and the
     * latency tail shortens while a small job still finishes in a few
     * launches. */
    uint32_t age_weight_us;
} msa_serve_config;

typedef struct msa_job_stats {
    double submit_ms;   /* host monotonic clock, ms */
    double admit_ms;
    double done_ms;
    uint64_t cells;
    uint32_t n;
    uint32_t launches;  /* merged launches this job's tiles were part of */
} msa_job_stats;

/* Starts a serving loop (continuous batching of all-pairs jobs): an
 * admission thread and a launch thread, each owning a context on the device.
 * No counterpart in the reference, which scores one database per process run
 * (src/museqa.cpp:223-236). Jobs are admitted in arrival order while their
 * device footprint fits the HBM budget; every merged launch takes tasks from
 * all admitted jobs, shared as batch_window_us says. */
int msa_serve_start(const msa_serve_config *cfg, msa_server **out);
/* Queues an all-pairs job (same inputs as msa_seqs_upload + table). */
int msa_serve_submit(msa_server *srv, const uint8_t *units, const uint64_t *offs,
                     const uint64_t *lens, uint32_t n, const msa_table *table,
                     uint64_t *job_id);
/* Waits up to timeout_ms (-1 = forever) for a job; copies n(n-1)/2 scores
 * (index i(i-1)/2+j, as msa_nw_all_pairs) into `out` and releases the job.
 * MSA_ERR_DEVICE_TIMEOUT if it is not done yet (the job stays queued). */
int msa_serve_wait(msa_server *srv, uint64_t job_id, int timeout_ms, int32_t *out,
                   msa_job_stats *stats);
int msa_serve_stop(msa_server *srv);

/* ------------------------------------------------------------ diagnostics */

/*
 * Throughput of one integer operation form (no counterpart in the reference;
 * it measures the INT32 issue roofline the NW kernels are reported against).
 * op: 0 IADD, 1 IMNMX, 2 viaddmax_s32, 3 vimax3_s32, 4 vadd2, 5 viaddmax_s16x2,
 * 6 vimax3_s16x2, 7 viaddmax_u16x2, 8 vimax3_u16x2, 9 vmaxu2, 10 PRMT,
 * 11 the 32-bit NW cell, 12 the signed 16x2 NW cell, 13 the biased 16x2 cell,
 * 14 the 16x2 cell on the gap-free state (vadd2 + vimax3_u16x2),
 * 15 shared-memory ld.shared.v4 bandwidth (ops_per_clk_sm = bytes per SM per clock).
 */
typedef struct msa_op_probe {
    double ops_per_clk_sm;  /* lane-operations per SM per SM clock */
    double ms;              /* kernel time of the measured launch */
    uint64_t lane_ops;
    double sm_clock_mhz;    /* SM cycles / elapsed time during the launch */
} msa_op_probe;
int msa_probe_op(msa_ctx *ctx, int op, int iters, msa_op_probe *out);

#ifdef __cplusplus
}
#endif
#endif
