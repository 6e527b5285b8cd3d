// Neighbor-joining on the device, bit-exact with the reference's
// njoining::sequential<transform::symmetric> and
// njoining::sequential<transform::linear<2>>
// (src/phylogeny/njoining/impl/sequential.cpp:80-358).
//
// Layout. The reference keeps a packed symmetric matrix and, after every join,
// swaps the removed OTU y with logical 0 and deletes logical 0
// (src/phylogeny/matrix.cu:359-384, sequential.cpp:210-224); every index then
// shifts down by one, which is the order its first-maximum tie-break scans in.
// Here D is a full n x n float matrix with row pitch P (a multiple of 4) and, at
// join number t, logical index k lives in physical slot t + k. Deleting logical
// 0 is the increment of t; the swap is one row and one column copy from slot t
// into slot t + y. Each row of the logical lower triangle is therefore one
// contiguous run of memory, read with 16-byte loads.
//
// The linear order (sequential.cpp:189-203) instead swaps y with the last
// logical OTU c-1 and drops the last (matrix.cu:443-460 exchanges every
// off-diagonal pair; the diagonal is zero). No index moves: logical k stays in
// slot k (t = 0 throughout), and the swap is one row and one column copy from
// slot c-1 into slot y, or, when x itself was the last, the new node's row and
// column written into y.
//
// Schedule. One thread-block cluster of K CTAs (16 where the device allows,
// else fewer) runs every join. Hardware cluster barriers (release/acquire)
// split a join into phases:
//   scan   CTAs 0..K-2 search the logical lower triangle for the largest
//          Q = (c-2) D - S_i - S_j with its first row-major index; each CTA
//          holds its own copy of S in shared memory;
//   A      each CTA's candidate is stored into every CTA's shared memory;
//   join   every CTA reduces the candidates identically and computes the row
//          update (new distances, new row sums) for all c rows, so the copies
//          of S stay equal without any exchange;
//   B      every read of rows x, y and 0 is done;
//   write  CTAs 0..K-2 write row and column x and copy logical 0 into y, while
//          the next scan already runs: that scan reads none of those cells
//          (see `pend` and `moved` in the kernel).
// The new node's row sum is a serial float fold over the c updates
// (sequential.cpp:259), the one sequential piece of a join. CTA K-1 computes
// it while the others scan the next join, skipping the new node's row and
// column; CTA K-1 then scans that row and column itself. Every float and double
// operation is written with an explicit rounding intrinsic in the reference's
// order, so no FMA contraction or reassociation can change a bit.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include <cooperative_groups.h>

#include "msa_internal.hpp"

namespace msa {
namespace njdev {

namespace cg = cooperative_groups;

constexpr unsigned kFull = 0xffffffffu;
constexpr int kThreads = 1024;
constexpr int kWarps = kThreads / 32;
constexpr unsigned kMaxCluster = 16;
constexpr uint32_t kNone = 0xffffffffu;
// Row chunks (4 floats) each lane has in flight while scanning.
constexpr int kBatch = 4;
// Phase counters: CTA 0 (scan, wait at A, join, wait at B, writes) and the
// folding CTA (fold, scan of the new node's row, wait at A).
constexpr int kCycleSlots = 8;

// Orderable key of a finite or +inf Q value; 0 for NaN and -inf, which the
// reference's strict `q > best` (best starting at -inf) never selects.
// -0 and +0 compare equal there, so both map to the +0 key.
__device__ __forceinline__ uint32_t order_key(float q)
{
    if(q != q || q == -INFINITY) return 0u;
    uint32_t b = __float_as_uint(q);
    if(b == 0x80000000u) b = 0u;
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// Two float lanes in one 64-bit register and the packed float operations of
// sm_100 on them: each lane is rounded to nearest as the scalar operation
// (no flush to zero), so `sub2(sub2(mul2(a, b), c), d)` gives per lane the
// bits of __fsub_rn(__fsub_rn(__fmul_rn(a, b), c), d) with half the issues.
__device__ __forceinline__ unsigned long long f2(float a, float b)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2_split(unsigned long long v, float &a, float &b)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ unsigned long long mul2(unsigned long long a, unsigned long long b)
{
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long sub2(unsigned long long a, unsigned long long b)
{
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

// A candidate pair (i, j), j < i, as one 64-bit key: larger Q wins; on equal
// Q the pair earlier in the reference's row-major scan of the lower triangle
// (smaller i, then smaller j) wins, which is the order of i << 16 | j (i, j <
// 2^16). 0 means "no candidate"; the low word names the pair.
__device__ __forceinline__ unsigned long long pack(uint32_t key, uint32_t i, uint32_t j)
{
    return key ? (((unsigned long long) key << 32) | (0xffffffffu - ((i << 16) | j))) : 0ull;
}
__device__ __forceinline__ uint32_t pair_of(unsigned long long v) { return 0xffffffffu - (uint32_t) v; }

__device__ __forceinline__ unsigned long long umax64(unsigned long long a, unsigned long long b) { return a > b ? a : b; }

// The warp's maximum of a 64-bit key in two 32-bit warp reductions: the
// largest high word, then the largest low word among the lanes holding it.
__device__ __forceinline__ unsigned long long warp_max(unsigned long long v)
{
    const uint32_t hi = (uint32_t) (v >> 32), lo = (uint32_t) v;
    const uint32_t mhi = __reduce_max_sync(kFull, hi);
    const uint32_t mlo = __reduce_max_sync(kFull, hi == mhi ? lo : 0u);
    return ((unsigned long long) mhi << 32) | mlo;
}

__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }

struct State {
    float *D;                  // n rows of P floats; slot t + k holds logical k
    const float *S0;           // initial row sums by slot
    uint32_t *rec_x, *rec_y;   // logical indices joined at each step
    float *rec_dx, *rec_dy;
    int *err;                  // 2: no joinable pair; 3: a wait between clusters ran out; 4: an invalid pair
    unsigned long long *cycles;   // kCycleSlots phase counters
    uint32_t n, P;
    // Helper clusters (clusters 1.. of the launch) scan a share of the rows
    // while the OTU count exceeds helper_c; cluster 0 joins. Zero-filled
    // before the launch.
    uint32_t helper_ctas;      // CTAs of all helper clusters (0: cluster 0 alone)
    uint32_t helper_c;
    float *s_pub;              // [2][P] row sums published by the folding CTA after a join
    uint32_t *pub_xy;          // [2] the join (x << 16 | y) they follow
    uint32_t *pub_seq;         // join number + 1 of the last publication; kStop ends the helpers
    unsigned long long *cand;  // [2][helper_ctas] each helper CTA's candidate key
    uint32_t *cand_seq;        // [helper_ctas] join number + 1 of its last candidate
    unsigned long long wait_ns;   // limit of every wait between clusters
    int stall_publication;     // test hook: the folding CTA never publishes
};

constexpr uint32_t kStop = 0xffffffffu;
// Helper clusters: at most this many CTAs in all; kDefaultClusters - 1 of
// them by default (none: on 2,000 OTUs, 3 helper clusters above 1,400 OTUs
// measured 21.65 ms against 21.64 ms for one cluster, because the two
// handoffs through global memory per join cost what the wider scan saves),
// scanning while more than kHelperMinCount OTUs remain; every wait between
// clusters ends after kWaitUs.
constexpr uint32_t kMaxHelperCtas = 128;
constexpr uint32_t kDefaultClusters = 1;
constexpr uint32_t kHelperMinCount = 1400;
constexpr uint32_t kWaitUs = 1000000;

// Release/acquire flags between clusters (gpu scope) and the global timer
// that bounds every wait on them.
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t *p, uint32_t v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Waits until *flag >= want; returns the value seen, or 0 when `limit_ns`
// passed first (the caller reports the timeout and stops waiting).
__device__ __forceinline__ uint32_t wait_flag(const uint32_t *flag, uint32_t want, unsigned long long limit_ns)
{
    const unsigned long long t0 = global_ns();
    for(;;) {
        const uint32_t v = ld_acquire(flag);
        if(v >= want) return v;
        if(global_ns() - t0 > limit_ns) return 0u;
        __nanosleep(128);
    }
}

// One scanning warp's share of a join's search (the kernel's scan phase):
// rows i = c-1 down to 1 of the logical lower triangle, longest first, warp
// gw of W taking places gw and 2W-1-gw of every 2W, so long and short rows
// pair up and the last, partial 2W hold the shortest rows. Warp `warp` of
// scanning CTA `s` (of `ns`) is gw = warp * ns + s, so consecutive places
// fall in different CTAs and the partial block spreads over all of them
// (with rows ascending and gw = s * 32 + warp, the longest leftover rows all
// fell to the first CTAs). The CTA's copy of
// S holds +inf in the dropped slots (< t), in `moved`'s slot and in the new
// node's (`pend`), so those columns give Q = -inf or NaN and never win; only
// the cells past a row's end are masked. Each lane keeps, per row, the largest
// chunk maximum and the first chunk reaching it, and its best over rows by
// (Q, row, chunk), which orders like the row-major index; the element inside
// the winning chunk is resolved once, after the scan. `moved`'s column of
// later rows is read from where its data still is (slot mslot): lane r loads
// it for the warp's r-th row before the row loop and offers it after, so the
// load waits in the shadow of the scan. The lane's best candidate goes into
// `best`.
struct ScanView {
    const float *D;   // slot t + k holds logical k; row pitch P
    const float *S;   // this CTA's row sums by slot
    uint32_t P, t, c, pend, moved, mslot;
    float cm2, s_moved;
};

template <bool TailCut>
__device__ __forceinline__ void scan_rows(const ScanView &v, uint32_t s, uint32_t ns, int warp, int lane,
                                          unsigned long long &best)
{
    const uint32_t W = ns * kWarps, gw = (uint32_t) warp * ns + s;
    const uint32_t base4 = v.t & ~3u;
    const float s_moved = v.s_moved;
    const unsigned long long cm2x2 = f2(v.cm2, v.cm2);
    auto row_of = [&](uint32_t i) { return v.D + (size_t) (i == v.moved ? v.mslot : v.t + i) * v.P + base4; };
    // Q = (c-2) * D - S_i - S_j for the four cells of a chunk, two per packed
    // operation; cells at or past the row's end (column hi) get -inf.
    auto chunk_raw = [&](const float4 &d, uint32_t col, unsigned long long si2, float &q0, float &q1, float &q2,
                         float &q3) {
        const float4 s = *reinterpret_cast<const float4 *>(v.S + col);
        f2_split(sub2(sub2(mul2(cm2x2, f2(d.x, d.y)), si2), f2(s.x, s.y)), q0, q1);
        f2_split(sub2(sub2(mul2(cm2x2, f2(d.z, d.w)), si2), f2(s.z, s.w)), q2, q3);
    };
    auto chunk_q = [&](const float4 &d, uint32_t col, uint32_t hi, unsigned long long si2, float &q0, float &q1,
                       float &q2, float &q3) {
        chunk_raw(d, col, si2, q0, q1, q2, q3);
        if(col + 4 > hi) {
            if(col >= hi) q0 = -INFINITY;
            if(col + 1 >= hi) q1 = -INFINITY;
            if(col + 2 >= hi) q2 = -INFINITY;
            if(col + 3 >= hi) q3 = -INFINITY;
        }
    };
    // The row of the warp's place p (p = 0 is row c-1), or 0 past the end.
    auto row_at = [&](uint32_t p) { return p + 1 < v.c ? v.c - 1 - p : 0u; };
    // The warp's r-th row (r = 2 * block + half), 0 when it has none or when
    // column `v.moved` of it is not read here.
    auto moved_row = [&](uint32_t r) {
        const uint32_t i = row_at((r >> 1) * 2 * W + ((r & 1) ? 2 * W - 1 - gw : gw));
        return (i <= v.moved || i == v.pend) ? 0u : i;
    };
    // Column `v.moved` of the warp's r-th row, for r = lane (with 15 scanning
    // CTAs a warp has at most 2 * ceil(12800 / 960) = 28 rows; any beyond 32
    // are read after the scan), from where logical 0's data still is.
    uint32_t mi = 0;
    float mq = 0.0f;
    if(v.moved != kNone) {
        mi = moved_row((uint32_t) lane);
        if(mi) mq = __ldcg(v.D + (size_t) (v.t + mi) * v.P + v.mslot);
    }
    unsigned long long lbest = 0;   // (key << 32) | ~(row << 14 | chunk)
    for(uint32_t base = 0; base + 1 < v.c; base += 2 * W) {
#pragma unroll 1
        for(int h = 0; h < 2; ++h) {
            const uint32_t i = row_at(base + (h ? 2 * W - 1 - gw : gw));
            if(i == 0 || i == v.pend) continue;
            const uint32_t hi = v.t + i;
            const float *row = row_of(i);
            const float si = i == v.moved ? s_moved : v.S[v.t + i];
            const unsigned long long si2 = f2(si, si);
            const uint32_t nch = (hi - base4 + 3) >> 2;
            float bq = -INFINITY;
            uint32_t bg = 0;
            // The row's last chunk, when it holds cells past the row's end:
            // chunk nfull, in lane nfull % 32's slot (nfull % span) / 32 of
            // the pass starting at g0 = tail_g0 (a pass spans 32 kBatch chunks).
            constexpr uint32_t span = 32 * kBatch;
            const uint32_t nfull = (hi - base4) >> 2, rem = (hi - base4) & 3u;
            const uint32_t tail_g0 = (TailCut && rem && (nfull & 31u) == (uint32_t) lane)
                                         ? nfull / span * span + (nfull & 31u)
                                         : 0xffffffffu;
            for(uint32_t g0 = lane; g0 < nch; g0 += 32 * kBatch) {
                float4 d[kBatch];
#pragma unroll
                for(int u = 0; u < kBatch; ++u)
                    if(g0 + 32 * u < nch) d[u] = __ldcg(reinterpret_cast<const float4 *>(row + 4 * (g0 + 32 * u)));
                if(TailCut && g0 == tail_g0) {
                    // D = -inf past the row's end gives Q = -inf there (NaN
                    // when c = 2), which never wins.
                    const uint32_t tu = (nfull % span) >> 5;
#pragma unroll
                    for(int u = 0; u < kBatch; ++u)
                        if((uint32_t) u == tu) {
                            d[u].w = -INFINITY;
                            if(rem <= 2) d[u].z = -INFINITY;
                            if(rem <= 1) d[u].y = -INFINITY;
                        }
                }
#pragma unroll
                for(int u = 0; u < kBatch; ++u) {
                    const uint32_t g = g0 + 32 * u;
                    if(g < nch) {
                        float q0, q1, q2, q3;
                        if constexpr(TailCut)
                            chunk_raw(d[u], base4 + 4 * g, si2, q0, q1, q2, q3);
                        else
                            chunk_q(d[u], base4 + 4 * g, hi, si2, q0, q1, q2, q3);
                        const float m = fmaxf(fmaxf(q0, q1), fmaxf(q2, q3));
                        if(m > bq) {
                            bq = m;
                            bg = g;
                        }
                    }
                }
            }
            const uint32_t key = order_key(bq);
            if(key) lbest = umax64(lbest, ((unsigned long long) key << 32) | (0xffffffffu - ((i << 14) | bg)));
        }
    }
    if(v.moved != kNone) {
        for(uint32_t r = (uint32_t) lane;;) {
            if(mi) {
                const float q = __fsub_rn(__fsub_rn(__fmul_rn(v.cm2, mq), v.S[v.t + mi]), s_moved);
                best = umax64(best, pack(order_key(q), mi, v.moved));
            }
            r += 32;
            // The warp has 2 ceil((c-1) / 2W) places: r is past them once its
            // block of 2W places starts at or after row c-1's place count.
            if((r >> 1) * 2 * W >= v.c - 1) break;
            mi = moved_row(r);
            if(mi) mq = __ldcg(v.D + (size_t) (v.t + mi) * v.P + v.mslot);
        }
    }
    if(lbest) {
        const uint32_t tail = 0xffffffffu - (uint32_t) (lbest & 0xffffffffull);
        const uint32_t i = tail >> 14, g = tail & 0x3fffu, col = base4 + 4 * g;
        const float si = i == v.moved ? s_moved : v.S[v.t + i];
        float q[4];
        chunk_q(__ldcg(reinterpret_cast<const float4 *>(row_of(i) + 4 * g)), col, v.t + i, f2(si, si), q[0], q[1],
                q[2], q[3]);
        const uint32_t key = (uint32_t) (lbest >> 32);
        int k = 3;
        if(order_key(q[2]) == key) k = 2;   // keep the first element equal to the maximum
        if(order_key(q[1]) == key) k = 1;
        if(order_key(q[0]) == key) k = 0;
        const uint32_t j = col + k - v.t;
        best = umax64(best, pack(key, i, j));
    }
}

// A helper CTA (clusters 1.. of the launch): scans its share of the rows of
// every join while the OTU count exceeds helper_c, with the same removal
// bookkeeping as cluster 0, and hands its best candidate to cluster 0's CTA 0.
// It starts from the initial row sums; after each join it takes the row sums
// and the joined pair that the folding CTA publishes (double-buffered by
// join parity) and masks them as the scanning CTAs of cluster 0 do. `sidx`
// is its place among all scanning CTAs (cluster 0's come first), `nscan` the
// number of them. Every wait is bounded by st.wait_ns; a wait
// that runs out sets err = 3 and ends the helper.
template <bool Linear>
__device__ void nj_helper(const State &st, float *S, uint32_t hidx, uint32_t sidx, uint32_t nscan)
{
    __shared__ unsigned long long hbest[kWarps];
    __shared__ float h_moved;
    __shared__ int h_stop;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t n = st.n, P = st.P;
    for(uint32_t k = tid; k < P; k += kThreads) S[k] = k < n ? st.S0[k] : 0.0f;
    if(tid == 0) {
        h_moved = 0.0f;
        h_stop = 0;
    }
    __syncthreads();
    uint32_t c = n, t = 0, step = 0, pend = kNone, moved = kNone, mslot = 0;
    while(c > 1 && c > st.helper_c) {
        unsigned long long best = 0;
        scan_rows<!Linear>(ScanView{st.D, S, P, t, c, pend, moved, mslot, (float) (c - 2), h_moved}, sidx, nscan, warp,
                           lane,
                  best);
        {
            const unsigned long long wm = warp_max(best);
            if(lane == 0) hbest[warp] = wm;
        }
        __syncthreads();
        const uint32_t buf = step & 1u;
        if(warp == 0) {
            const unsigned long long v = lane < kWarps ? hbest[lane] : 0ull;
            const unsigned long long m = warp_max(v);
            if(lane == 0) {
                st.cand[(size_t) buf * st.helper_ctas + hidx] = m;
                st_release(st.cand_seq + hidx, step + 1);
            }
        }
        if(c - 1 <= st.helper_c) break;   // cluster 0 scans the next joins alone
        if(tid == 0) {
            const uint32_t v = wait_flag(st.pub_seq, step + 1, st.wait_ns);
            if(v == 0u) atomicExch(st.err, 3);
            h_stop = (v == 0u || v == kStop) ? 1 : 0;
        }
        __syncthreads();
        if(h_stop) break;
        // The join cluster 0 made, and its row sums after it.
        const uint32_t xy = __ldcg(st.pub_xy + buf);
        const uint32_t x = xy >> 16, y = xy & 0xffffu;
        if(x >= c || y >= x) {   // never a pair of this join
            if(tid == 0) atomicExch(st.err, 4);
            break;
        }
        const float *pub = st.s_pub + (size_t) buf * P;
        // Slots [t, t + c) only: those below t were dropped and keep the +inf
        // that masks them in the scan's first chunk (from slot t & ~3).
        for(uint32_t k = t + tid; k < t + c; k += kThreads) S[k] = __ldcg(pub + k);
        __syncthreads();
        const bool mv = Linear ? x != c - 1 : y != 0;
        if(tid == 0) {
            // As the scanning CTAs of cluster 0 (update_cache): the moved
            // data's row sum aside, +inf in its slot, in a dropped slot and
            // in the new node's (published before its fold).
            if(mv) {
                h_moved = S[t + y];
                S[t + y] = INFINITY;
            }
            if(!Linear) S[t] = INFINITY;
            S[Linear && !mv ? y : t + x] = INFINITY;   // the new node's slot
        }
        if(Linear) {
            pend = mv ? x : y;
            moved = mv ? y : kNone;
            mslot = c - 1;
        } else {
            pend = x - 1;
            moved = y != 0 ? y - 1 : kNone;
            mslot = t;
            ++t;
        }
        ++step;
        --c;
        __syncthreads();
    }
}

// kHelp: the launch has helper clusters (compiled separately, so that the
// one-cluster kernel carries none of their code).
template <bool Linear, bool kHelp>
__global__ void __launch_bounds__(kThreads, 1) nj_cluster_kernel(State st)
{
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t n = st.n, P = st.P;
    // Shared layout: S by slot, new distances ND and double updates U by
    // logical index (all P entries long; P is a multiple of 4).
    float *S = reinterpret_cast<float *>(smem_raw);
    float *ND = S + P;
    double *U = reinterpret_cast<double *>(smem_raw + (size_t) 8 * P);
    // Each CTA's best key, written into every CTA before barrier A.
    __shared__ unsigned long long parts[kMaxCluster];
    __shared__ unsigned long long wbest[kWarps];
    // Phase cycle counters live in shared memory, leaving registers to the
    // scan's loads in flight.
    __shared__ unsigned long long cyc[kCycleSlots];
    // Row sum of `moved` while this CTA's S holds +inf in its slot (CTAs 0..F-1).
    __shared__ float s_moved_sh;
    // Row sum of the new node `pend`, written here by CTA F after its fold,
    // while this CTA's S holds +inf in its slot (CTAs 0..F-1).
    __shared__ float s_pend_sh;
    // A scanning CTA r's slice of the join, [c r / F, c (r + 1) / F), kept as
    // quotients and remainders (q F + rem = c m for m = r and r + 1) that
    // the CTA's last thread steps down with c, so that no join divides.
    __shared__ uint32_t sl_q[2], sl_rem[2];

    const unsigned K = cluster.num_blocks();
    const unsigned rank = cluster.block_rank();
    const unsigned F = K - 1;   // the CTA that folds new row sums
    if constexpr(kHelp) {
        if(blockIdx.x >= K) {       // a helper cluster
            nj_helper<Linear>(st, reinterpret_cast<float *>(smem_raw), blockIdx.x - K, F + blockIdx.x - K,
                              F + st.helper_ctas);
            return;
        }
    }
    const bool folder = rank == F;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float *D = st.D;
    // Set (in every CTA of cluster 0, before barrier A) once a wait for the
    // helpers ran out: cluster 0 then scans alone.
    __shared__ int hoff;
    const bool timer = tid == 0 && (rank == 0 || folder);
    if(tid < kCycleSlots) cyc[tid] = 0;
    if(tid == 0) {
        s_moved_sh = 0.0f;
        s_pend_sh = 0.0f;
        hoff = 0;
        for(int h = 0; h < 2; ++h) {
            sl_q[h] = n * (rank + h) / F;
            sl_rem[h] = n * (rank + h) % F;
        }
    }
    unsigned long long t_last = clock64();
    auto mark = [&](int k) {
        const unsigned long long now = clock64();
        cyc[k] += now - t_last;
        t_last = now;
    };

    for(uint32_t k = tid; k < P; k += kThreads) {
        S[k] = k < n ? st.S0[k] : 0.0f;
        ND[k] = 0.0f;
    }
    cluster.sync();   // every CTA is running before any shared-memory exchange

    uint32_t c = n, t = 0, step = 0;
    // Logical indices (in the current window) that the previous join left
    // unfinished: `pend` is the new node, whose row sum CTA F is still folding
    // and whose row and column only CTA F scans (from ND); `moved` took logical
    // 0's data, which the previous join's writes may not have copied yet, so
    // scans read it where it was (slot t - 1): its row there, and column t - 1
    // of every later row.
    // `mslot` is the slot where `moved`'s data still is.
    uint32_t pend = kNone, moved = kNone, mslot = 0;
    bool failed = false, bad = false;

    while(c > 1) {
        const float cm2 = (float) (c - 2);
        // The helper clusters scan with cluster 0 for this join.
        const bool helped = kHelp && st.helper_ctas != 0u && !hoff && c > st.helper_c;
        unsigned long long best = 0;

        // ---- scan
        if(!folder) {
            // This CTA's share of the rows of the logical lower triangle
            // (scan_rows), with +inf in S masking the dropped slots and those
            // of `moved` and the new node.
            scan_rows<!Linear>(ScanView{D, S, P, t, c, pend, moved, mslot, cm2, s_moved_sh}, rank,
                      F + (helped ? st.helper_ctas : 0u), warp, lane, best);
        } else if(pend != kNone) {
            // The new node's row and column, from the distances the last join
            // computed (ND, indexed by that join's logical order: logical j
            // was j + 1 there in the symmetric order, j in the linear one, and
            // `moved` was 0 or the last): pairs (pend, j < pend) and
            // (j > pend, pend) with the reference's operand order for each.
            const uint32_t x = pend;
            const float sx = S[t + x];
            for(uint32_t j = tid; j < c; j += kThreads) {
                if(j == x) continue;
                const float d = ND[j == moved ? (Linear ? mslot : 0u) : (Linear ? j : j + 1)];
                const float sj = S[t + j];
                if(j < x) {
                    const float q = __fsub_rn(__fsub_rn(__fmul_rn(cm2, d), sx), sj);
                    best = umax64(best, pack(order_key(q), x, j));
                } else {
                    const float q = __fsub_rn(__fsub_rn(__fmul_rn(cm2, d), sj), sx);
                    best = umax64(best, pack(order_key(q), j, x));
                }
            }
        }
        // Keys are unique (distinct pairs) and name their pair, so the
        // maximum over all CTAs is the join.
        {
            const unsigned long long wm = warp_max(best);
            if(lane == 0) wbest[warp] = wm;
        }
        __syncthreads();
        if(warp == 0) {
            const unsigned long long v = lane < kWarps ? wbest[lane] : 0ull;
            unsigned long long m = warp_max(v);
            int off = 0;
            if(kHelp && rank == 0 && helped) {
                // The helper CTAs' candidates for this join, each lane waiting
                // for its share of them; merged into this CTA's part.
                const uint32_t buf = step & 1u;
                unsigned long long hb = 0;
                bool ok = true;
                for(uint32_t h = lane; h < st.helper_ctas; h += 32) {
                    if(ok && wait_flag(st.cand_seq + h, step + 1, st.wait_ns) != 0u)
                        hb = umax64(hb, __ldcg(st.cand + (size_t) buf * st.helper_ctas + h));
                    else
                        ok = false;
                }
                m = umax64(m, warp_max(hb));
                if(!__all_sync(kFull, ok)) {
                    off = 1;
                    if(lane == 0) atomicExch(st.err, 3);
                }
            }
            if((unsigned) lane < K) {
                cluster.map_shared_rank(parts, (unsigned) lane)[rank] = m;
                if(off) cluster.map_shared_rank(&hoff, (unsigned) lane)[0] = 1;
            }
        }
        if(timer) mark(rank == 0 ? 0 : 6);
        cluster_arrive();   // A
        cluster_wait();
        if(timer) mark(rank == 0 ? 1 : 7);

        // ---- join
        // Every warp reduces the K parts itself (lane r reads part r).
        const unsigned long long win = warp_max((unsigned) lane < K ? parts[lane] : 0ull);
        if(win == 0ull) {   // no selectable Q (all NaN): the reference would index an undefined pair
            failed = true;
            break;
        }
        const uint32_t x = pair_of(win) >> 16, y = pair_of(win) & 0xffffu;
        if(x >= c || y >= x) {   // never a pair of this join: report it, touch nothing
            bad = true;
            break;
        }
        // The logical index whose data takes y's place (0, or the last in the
        // linear order), and whether there is such a move: none when y is 0
        // (symmetric), or when x itself is the last (linear; the new node then
        // takes y's place).
        const uint32_t src = Linear ? c - 1 : 0u;
        const bool mv = Linear ? x != c - 1 : y != 0;
        const float *rx = D + (size_t) (t + x) * P + t;
        const float *ry = D + (size_t) (t + y) * P + t;
        const float *r0 = D + (size_t) (t + src) * P + t;
        const float dxy = __ldcg(rx + y);
        const uint32_t nslot = Linear && !mv ? y : t + x;
        // Row sums of the new node and of the moved data, held aside while a
        // scanning CTA's S has +inf in their slots.
        const float s_moved = s_moved_sh, s_pend = s_pend_sh;

        if(folder) {
            // CTA F computes the whole join for its own S, ND and U (the fold
            // needs all of them), but only its reads of rows x and y come
            // before barrier B (the writes after B change those rows): it
            // keeps D[x][i] + D[y][i] in ND, arrives, and finishes after.
            for(uint32_t i = tid; i < c; i += kThreads) ND[i] = __fadd_rn(__ldcg(rx + i), __ldcg(ry + i));
            cluster_arrive();   // B
            // join_pair (sequential.cpp:247-267); i = x and i = y read the
            // diagonal and D[x][y], as the reference does. S has no masks here.
            // The thread of element y also computes raise_candidate.
            bool exact = true;
            for(uint32_t i = tid; i < c; i += kThreads) {
                const float prev = ND[i];
                const double u = __dmul_rn((double) __fsub_rn(prev, dxy), 0.5);
                const float nd = __double2float_rn(u);
                U[i] = u;
                ND[i] = nd;
                exact = exact && ((double) nd == u);
                const float s_old = S[t + i];
                if(i == y) {
                    // raise_candidate (sequential.cpp:142-152) from the row
                    // sums before this join's update (S[x] is not updated
                    // here, S[y] is read before it is).
                    const float pairsum = __fsub_rn(S[t + x], s_old);
                    const float den = (float) (2u * (c - 2));
                    const float q = __fdiv_rn(pairsum, den);
                    float dx = __double2float_rn(__dadd_rn(__dmul_rn(0.5, (double) dxy), (double) q));
                    float dy = __fsub_rn(dxy, dx);
                    // The last join divides by 2(c-2) = 0; for 0/0 the
                    // reference's x86 SSE arithmetic yields the default NaN
                    // 0xFFC00000 and propagates it into dx and dy, where the
                    // GPU would give its canonical 0x7FFFFFFF.
                    if(dx != dx) dx = __uint_as_float(0xFFC00000u);
                    if(dy != dy) dy = __uint_as_float(0xFFC00000u);
                    st.rec_x[step] = x;
                    st.rec_y[step] = y;
                    st.rec_dx[step] = dx;
                    st.rec_dy[step] = dy;
                }
                if(i != x) S[t + i] = __double2float_rn(__dadd_rn((double) s_old, __dsub_rn(u, (double) prev)));
            }
            exact = __syncthreads_and(exact);
            // update_cache (sequential.cpp:189-224): logical `src` takes y's place.
            if(tid == 0 && mv) S[t + y] = S[t + src];
            // The row sums after this join and the joined pair, for the helper
            // clusters' next scan (this CTA's copy has no +inf masks).
            if(kHelp && st.helper_ctas != 0u && !hoff && c - 1 > st.helper_c) {
                __syncthreads();   // update_cache above
                const uint32_t buf = step & 1u;
                float *pub = st.s_pub + (size_t) buf * P;
                for(uint32_t k = t + tid; k < t + c; k += kThreads) __stcg(pub + k, S[k]);
                if(tid == 0) st.pub_xy[buf] = (x << 16) | y;
                __syncthreads();
                if(tid == 0 && !st.stall_publication) {
                    __threadfence();
                    st_release(st.pub_seq, step + 1);
                }
            }
            // Serial fold of the new row sum, i ascending. When every update is
            // a float value, the double add rounded to float equals a float add
            // (double has >= 2*24+2 significand bits), so the short float chain
            // is used; otherwise the literal double one. Warp 0 runs it (every
            // lane the same chain, reading ND by broadcast 16-byte loads that
            // do not depend on the chain); ND and U were written before the
            // __syncthreads_and above. The sum goes to the other CTAs after B,
            // when none of them still reads s_pend_sh for this join.
            float ns = 0.0f;
            if(warp == 0) {
                const unsigned long long f0 = clock64();
                if(exact) {
                    const uint32_t c4 = c & ~3u;
#pragma unroll 8
                    for(uint32_t i = 0; i < c4; i += 4) {
                        const float4 v = *reinterpret_cast<const float4 *>(ND + i);
                        ns = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(ns, v.x), v.y), v.z), v.w);
                    }
                    for(uint32_t i = c4; i < c; ++i) ns = __fadd_rn(ns, ND[i]);
                } else {
                    for(uint32_t i = 0; i < c; ++i) ns = __double2float_rn(__dadd_rn((double) ns, U[i]));
                }
                if(lane == 0) cyc[5] += clock64() - f0;
            }
            cluster_wait();
            if(warp == 0) {
                if((unsigned) lane == F)
                    S[nslot] = ns;
                else if((unsigned) lane < K)
                    *cluster.map_shared_rank(&s_pend_sh, (unsigned) lane) = ns;
            }
            __syncthreads();   // the folded row sum is in this CTA's S
            if(timer) t_last = clock64();
        } else {
            // The scanning CTAs split the join: CTA r < F takes the elements
            // [c r / F, c (r + 1) / F), the slice it also writes back after B.
            // The loads of a thread's first element are issued here, and the
            // moved row's entry too, so the writes wait for no load.
            const uint32_t jlo = sl_q[0], jhi = sl_q[1];
            const uint32_t ji = jlo + tid;
            float a0 = ji < jhi ? __ldcg(rx + ji) : 0.0f, b0 = ji < jhi ? __ldcg(ry + ji) : 0.0f;
            const float v0 = (ji < jhi && mv) ? __ldcg(r0 + ji) : 0.0f;
            // The thread of element x also writes src's new distance into
            // D[x][y] and D[y][x], and the thread of element y src's diagonal
            // into D[y][y]: their reads (none of those cells is written by
            // this join) are issued here with the slice's, not after B.
            float px = 0.0f, py = 0.0f;
            if(mv && ji == x) {
                px = __ldcg(rx + src);
                py = __ldcg(ry + src);
            }
            if(mv && ji == y) px = __ldcg(r0 + src);
            auto s_of = [&](uint32_t i) { return i == moved ? s_moved : i == pend ? s_pend : S[t + i]; };

            // join_pair (sequential.cpp:247-267) on the slice. D[i][x] and
            // D[i][y] are read as row x and row y (the matrix is symmetric bit
            // for bit); i = x and i = y read the diagonal and D[x][y], as the
            // reference does. Each new row sum goes into every scanning CTA's
            // S (CTA F computes raise_candidate in its copy of the join).
            for(uint32_t i = ji; i < jhi; i += kThreads) {
                const uint32_t in = i + kThreads;
                const float an = in < jhi ? __ldcg(rx + in) : 0.0f, bn = in < jhi ? __ldcg(ry + in) : 0.0f;
                const float prev = __fadd_rn(a0, b0);
                const double u = __dmul_rn((double) __fsub_rn(prev, dxy), 0.5);
                ND[i] = __double2float_rn(u);
                const float s_old = s_of(i);
                if(i != x) {
                    const float sn = __double2float_rn(__dadd_rn((double) s_old, __dsub_rn(u, (double) prev)));
                    for(unsigned r = 0; r < F; ++r) cluster.map_shared_rank(S, r)[t + i] = sn;
                }
                a0 = an;
                b0 = bn;
            }
            if(timer && rank == 0) mark(2);
            // B: every read of rows x, y and the moved row is done, and every
            // slice's row sums are in every scanning CTA's S.
            cluster_arrive();
            cluster_wait();
            if(timer) mark(3);
            // update_cache (sequential.cpp:189-224): logical `src` takes y's
            // place. Keep that row sum aside and put +inf in its slot, in
            // logical 0's (symmetric: dropped next) and in the new node's slot
            // `nslot` (x's, or y's when the new node takes y's place), for the
            // next scan. The linear order's dropped slot c-1 lies past every
            // row the next scan reads. The new node's folded sum arrives in
            // s_pend_sh; the next join writes every slot but x's from the sums
            // it read, so a +inf slot ends up with its sum unless it is masked
            // again. The CTA's last thread does it (and steps the slice down
            // below): in a 16-CTA cluster it holds no element of the slice
            // (at most 854 at n <= 12800), so the threads that write wait for
            // neither (with fewer CTAs it may also write, after the masks).
            if(tid == kThreads - 1) {
                if(mv) {
                    s_moved_sh = S[t + src];
                    S[t + y] = INFINITY;
                }
                if(!Linear) S[t] = INFINITY;
                S[nslot] = INFINITY;
            }
            // The writes of this CTA's slice, after B, overlapping the next
            // scan (which skips the new node's row, reads the moved data where
            // it was, and masks columns x and y): row and column x get the new
            // distances, and logical `src`'s row and column move into y (or,
            // in the linear order when x is the last, the new distances go
            // into y). D[x][y] and D[y][x] take src's new distance, which the
            // thread of element x computes itself from its own reads.
            float *wx = D + (size_t) (t + x) * P + t;
            float *wy = D + (size_t) (t + y) * P + t;
            for(uint32_t i = ji; i < jhi; i += kThreads) {
                if(Linear && !mv) {
                    if(i == y || i == x) continue;
                    const float nd = ND[i];
                    __stcg(wy + i, nd);
                    __stcg(D + (size_t) i * P + y, nd);
                    continue;
                }
                if(i == src || (!Linear && y == 0 && i == y)) continue;
                if(i == y) {
                    __stcg(wy + y, i == ji ? px : __ldcg(r0 + src));   // src's diagonal
                    continue;
                }
                const float nd = ND[i];
                if(i == x) {
                    __stcg(wx + x, nd);
                    if(mv) {
                        // src's new distance, with the join's operations on
                        // the same operands (read before B).
                        const float ax = i == ji ? px : __ldcg(rx + src), ay = i == ji ? py : __ldcg(ry + src);
                        const float nds = __double2float_rn(__dmul_rn((double) __fsub_rn(__fadd_rn(ax, ay), dxy), 0.5));
                        __stcg(wx + y, nds);
                        __stcg(wy + x, nds);
                    }
                    continue;
                }
                __stcg(wx + i, nd);
                __stcg(D + (size_t) (t + i) * P + t + x, nd);
                if(mv) {
                    const float v = i == ji ? v0 : __ldcg(r0 + i);
                    __stcg(wy + i, v);
                    __stcg(D + (size_t) (t + i) * P + t + y, v);
                }
            }
            if(tid == kThreads - 1)   // the slice of the next join, with c - 1 OTUs
                for(int h = 0; h < 2; ++h) {
                    const uint32_t m = rank + h;
                    if(sl_rem[h] >= m) {
                        sl_rem[h] -= m;
                    } else {
                        sl_rem[h] += F - m;
                        --sl_q[h];
                    }
                }
            __syncthreads();   // the +inf masks above, before the scan
            if(timer) mark(4);
        }

        if(Linear) {
            // The last logical index leaves; the new node stays at x (or
            // takes y's place when x was the last) and the last one's data
            // moves to y.
            pend = mv ? x : y;
            moved = mv ? y : kNone;
            mslot = c - 1;
        } else {
            // Logical 0 leaves the window; the new node sits at x - 1 and
            // logical 0's data at y - 1.
            pend = x - 1;
            moved = y != 0 ? y - 1 : kNone;
            mslot = t;
            ++t;
        }
        ++step;
        --c;
    }
    if(failed && rank == 0 && tid == 0) atomicExch(st.err, 2);
    if(bad && rank == 0 && tid == 0) atomicExch(st.err, 4);
    // Helpers still waiting for a publication stop.
    if(kHelp && folder && tid == 0 && st.helper_ctas != 0u && !st.stall_publication) st_release(st.pub_seq, kStop);
    if(tid == 0 && rank == 0)
        for(int k = 0; k < 5; ++k) st.cycles[k] = cyc[k];
    if(tid == 0 && folder)
        for(int k = 5; k < kCycleSlots; ++k) st.cycles[k] = cyc[k];
    cluster.sync();   // no CTA leaves while another may still write its shared memory
}

// Packed triangle (float or int32) -> full symmetric matrix of pitch P,
// diagonal and padding 0.
template <class T>
__global__ void inflate_kernel(const T *__restrict__ tri, float *__restrict__ D, uint32_t n, uint32_t P)
{
    const uint64_t total = (uint64_t) n * P;
    for(uint64_t e = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t) gridDim.x * blockDim.x) {
        const uint64_t i = e / P, j = e - i * P;
        float v = 0.0f;
        if(j < n) {
            if(i > j) v = (float) tri[i * (i - 1) / 2 + j];
            else if(j > i) v = (float) tri[j * (j - 1) / 2 + i];
        }
        D[e] = v;
    }
}

// cache_init (sequential.cpp:80-94): S[k] folds D[k][j] over j != k ascending,
// from 0. Thread k reads column k (= row k by symmetry) so a warp's reads coalesce.
__global__ void row_sums_kernel(const float *__restrict__ D, float *__restrict__ S, uint32_t n, uint32_t P)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if(k >= n) return;
    float s = 0.0f;
    for(uint32_t j = 0; j < n; ++j)
        if(j != k) s = __fadd_rn(s, D[(size_t) j * P + k]);
    S[k] = s;
}

// Largest cluster (16, 8, 4 or 2 CTAs) that can be resident with `smem` bytes
// of dynamic shared memory per CTA; 0 if none.
template <bool Linear, bool kHelp>
unsigned pick_cluster(size_t smem)
{
    for(unsigned k : {16u, 8u, 4u, 2u}) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = k;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(k);
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = smem;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        if(cudaOccupancyMaxActiveClusters(&clusters, nj_cluster_kernel<Linear, kHelp>, &cfg) == cudaSuccess &&
           clusters >= 1)
            return k;
        cudaGetLastError();
    }
    return 0;
}

}  // namespace njdev

int nj_run(msa_ctx *ctx, const void *tri, int kind, uint32_t n, int order, msa_otu *out)
{
    const bool linear = order == MSA_NJ_LINEAR;
    auto kern_one = linear ? njdev::nj_cluster_kernel<true, false> : njdev::nj_cluster_kernel<false, false>;
    auto kern_help = linear ? njdev::nj_cluster_kernel<true, true> : njdev::nj_cluster_kernel<false, true>;
    cudaStream_t s = ctx->stream;
    const uint32_t P = (n + 3) & ~3u;
    const size_t smem = (size_t) P * 16;   // S, ND (4 B each), U (8 B)
    if(n > 12800) return set_error(ctx, MSA_ERR_TOO_LARGE, "neighbor-joining supports at most 12800 OTUs");
    const uint64_t ntri = (uint64_t) n * (n - 1) / 2;

    // Device layout.
    size_t off = 0;
    auto take = [&off](size_t b) { size_t o = off; off = round_up(off + b, 256); return o; };
    const size_t oD = take((size_t) n * P * 4), oS = take(n * 4), oRx = take(n * 4), oRy = take(n * 4),
                 oRdx = take(n * 4), oRdy = take(n * 4), oErr = take(64), oCyc = take(64),
                 oTri = take((kind == MSA_TRI_F32_HOST || kind == MSA_TRI_I32_HOST) ? ntri * 4 : 0),
                 oPub = take((size_t) 2 * P * 4),
                 // flags between clusters: pub_seq, pub_xy[2], cand_seq[], cand[][][2]
                 oSync = take(64 + (size_t) njdev::kMaxHelperCtas * 4),
                 oCand = take((size_t) 2 * njdev::kMaxHelperCtas * 16);
    MSA_CUDA_TRY(ctx, ctx->nj_buf.ensure(off));
    char *base = (char *) ctx->nj_buf.ptr;
    njdev::State st{};
    st.D = (float *) (base + oD);
    st.S0 = (const float *) (base + oS);
    st.rec_x = (uint32_t *) (base + oRx);
    st.rec_y = (uint32_t *) (base + oRy);
    st.rec_dx = (float *) (base + oRdx);
    st.rec_dy = (float *) (base + oRdy);
    st.err = (int *) (base + oErr);
    st.cycles = (unsigned long long *) (base + oCyc);
    st.n = n;
    st.P = P;

    for(auto kf : {kern_one, kern_help}) {
        MSA_CUDA_TRY(ctx, cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        MSA_CUDA_TRY(ctx, cudaFuncSetAttribute(kf, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    }
    const unsigned K = linear ? njdev::pick_cluster<true, false>(smem) : njdev::pick_cluster<false, false>(smem);
    if(K < 2) return set_error(ctx, MSA_ERR_CUDA, "neighbor-joining cluster cannot be resident");
    // Helper clusters: as many as can be resident beside cluster 0 (each on
    // its own GPC), at most the context's setting, and only when some join
    // has more OTUs than the helpers' threshold.
    const uint32_t helper_c = std::max<uint32_t>(ctx->nj_helper_c ? ctx->nj_helper_c : njdev::kHelperMinCount, 2);
    uint32_t clusters = 1;
    if(ctx->nj_clusters != 1 && n > helper_c + 1) {
        cudaLaunchConfig_t q = {};
        cudaLaunchAttribute qa[1];
        qa[0].id = cudaLaunchAttributeClusterDimension;
        qa[0].val.clusterDim.x = K;
        qa[0].val.clusterDim.y = 1;
        qa[0].val.clusterDim.z = 1;
        q.gridDim = dim3(K);
        q.blockDim = dim3(njdev::kThreads);
        q.dynamicSmemBytes = smem;
        q.attrs = qa;
        q.numAttrs = 1;
        int resident = 0;
        if(cudaOccupancyMaxActiveClusters(&resident, kern_help, &q) != cudaSuccess) {
            cudaGetLastError();
            resident = 1;
        }
        const uint32_t want = ctx->nj_clusters ? (uint32_t) ctx->nj_clusters : njdev::kDefaultClusters;
        clusters = std::max<uint32_t>(1, std::min<uint32_t>({want, (uint32_t) resident,
                                                              1 + njdev::kMaxHelperCtas / K}));
    }
    auto kern = clusters > 1 ? kern_help : kern_one;
    char *sync = base + oSync;
    st.helper_ctas = (clusters - 1) * K;
    st.helper_c = helper_c;
    st.s_pub = (float *) (base + oPub);
    st.pub_seq = (uint32_t *) sync;
    st.pub_xy = (uint32_t *) (sync + 16);
    st.cand_seq = (uint32_t *) (sync + 64);
    st.cand = (unsigned long long *) (base + oCand);
    st.wait_ns = (unsigned long long) (ctx->nj_wait_us ? ctx->nj_wait_us : njdev::kWaitUs) * 1000ull;
    st.stall_publication = ctx->nj_stall;

    MSA_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[0], s));
    const void *dtri = tri;
    if(kind == MSA_TRI_F32_HOST || kind == MSA_TRI_I32_HOST) {
        MSA_CUDA_TRY(ctx, cudaMemcpyAsync(base + oTri, tri, ntri * 4, cudaMemcpyHostToDevice, s));
        dtri = base + oTri;
    }
    const unsigned ib = (unsigned) std::min<uint64_t>(((uint64_t) n * P + 255) / 256, 65535);
    if(kind == MSA_TRI_F32_HOST || kind == MSA_TRI_F32_DEVICE)
        njdev::inflate_kernel<float><<<ib, 256, 0, s>>>((const float *) dtri, st.D, n, P);
    else
        njdev::inflate_kernel<int32_t><<<ib, 256, 0, s>>>((const int32_t *) dtri, st.D, n, P);
    MSA_CUDA_TRY(ctx, cudaGetLastError());
    njdev::row_sums_kernel<<<(n + 255) / 256, 256, 0, s>>>(st.D, (float *) (base + oS), n, P);
    MSA_CUDA_TRY(ctx, cudaGetLastError());
    MSA_CUDA_TRY(ctx, cudaMemsetAsync(base + oErr, 0, 64, s));
    // Joins the kernel never records stay invalid (0xffffffff) and are caught
    // before the tree is built.
    MSA_CUDA_TRY(ctx, cudaMemsetAsync(base + oRx, 0xff, (size_t) n * 4, s));
    MSA_CUDA_TRY(ctx, cudaMemsetAsync(base + oRy, 0xff, (size_t) n * 4, s));
    MSA_CUDA_TRY(ctx, cudaMemsetAsync(base + oCyc, 0, 64, s));
    MSA_CUDA_TRY(ctx, cudaMemsetAsync(sync, 0, 64 + (size_t) njdev::kMaxHelperCtas * 4, s));
    ctx->launches += 2;

    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = K;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(K * clusters);
    cfg.blockDim = dim3(njdev::kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    MSA_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[1], s));
    MSA_CUDA_TRY(ctx, cudaLaunchKernelEx(&cfg, kern, st));
    MSA_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[2], s));
    ctx->launches++;
    unsigned long long cyc[8] = {0, 0, 0, 0, 0, 0, 0, 0};

    std::vector<uint32_t> rx(n - 1), ry(n - 1);
    std::vector<float> rdx(n - 1), rdy(n - 1);
    int err = 0;
    MSA_CUDA_TRY(ctx, cudaMemcpyAsync(rx.data(), st.rec_x, (n - 1) * 4, cudaMemcpyDeviceToHost, s));
    MSA_CUDA_TRY(ctx, cudaMemcpyAsync(ry.data(), st.rec_y, (n - 1) * 4, cudaMemcpyDeviceToHost, s));
    MSA_CUDA_TRY(ctx, cudaMemcpyAsync(rdx.data(), st.rec_dx, (n - 1) * 4, cudaMemcpyDeviceToHost, s));
    MSA_CUDA_TRY(ctx, cudaMemcpyAsync(rdy.data(), st.rec_dy, (n - 1) * 4, cudaMemcpyDeviceToHost, s));
    MSA_CUDA_TRY(ctx, cudaMemcpyAsync(&err, st.err, 4, cudaMemcpyDeviceToHost, s));
    MSA_CUDA_TRY(ctx, cudaMemcpyAsync(cyc, st.cycles, sizeof(cyc), cudaMemcpyDeviceToHost, s));
    MSA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    {
        msa_nj_stats ns{};
        float ms = 0, ms_all = 0;
        cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]);
        cudaEventElapsedTime(&ms_all, ctx->ev[0], ctx->ev[2]);
        ns.kernel_ms = ms;
        ns.total_ms = ms_all;
        ns.n = n;
        ns.cluster = K;
        ns.helper_clusters = clusters - 1;
        ns.cycles_scan = cyc[0];
        ns.cycles_wait = cyc[1];
        ns.cycles_join = cyc[2];
        ns.cycles_join_wait = cyc[3];
        ns.cycles_write = cyc[4];
        ns.cycles_fold = cyc[5];
        ns.cycles_fold_row = cyc[6];
        ns.cycles_fold_wait = cyc[7];
        ctx->nj_last = ns;
    }
    if(err == 2) return set_error(ctx, MSA_ERR_UNDEFINED, "no joinable pair: every Q value is NaN");
    if(err == 4) return set_error(ctx, MSA_ERR_CUDA, "neighbor-joining chose a pair outside the matrix");
    if(err == 3)
        return set_error(ctx, MSA_ERR_DEVICE_TIMEOUT,
                         "a wait between the neighbor-joining clusters ran out; the tree was not built");

    for(uint32_t k = 0; k + 1 < n; ++k)
        if(rx[k] >= n - k || ry[k] >= rx[k])
            return set_error(ctx, MSA_ERR_CUDA, "neighbor-joining recorded an invalid join");

    // star tree (src/phylogeny/njoining/star.cuh:61-72). The kernel records
    // logical indices; the OTU in each slot follows the same moves (slot of x
    // gets the parent; logical 0's OTU, or in the linear order the last one's,
    // moves into y's slot).
    const uint32_t nodes = 2 * n - 1;
    for(uint32_t k = 0; k < nodes; ++k) {
        out[k].parent = out[k].child[0] = out[k].child[1] = 0xffffffffu;
        out[k].distance = FLT_MAX;
        out[k].level = 0;
    }
    std::vector<uint32_t> map(n);
    for(uint32_t k = 0; k < n; ++k) map[k] = k;
    for(uint32_t k = 0; k + 1 < n; ++k) {
        const uint32_t parent = n + k;
        uint32_t a, b;
        if(linear) {
            // sequential.cpp:273 then :201-202.
            const uint32_t c = n - k;
            a = map[rx[k]];
            b = map[ry[k]];
            map[rx[k]] = parent;
            std::swap(map[ry[k]], map[c - 1]);
        } else {
            a = map[k + rx[k]];
            b = map[k + ry[k]];
            map[k + rx[k]] = parent;
            if(ry[k] != 0) map[k + ry[k]] = map[k];
        }
        const uint32_t c1 = a < b ? a : b, c2 = a < b ? b : a;
        const float d1 = a < b ? rdx[k] : rdy[k], d2 = a < b ? rdy[k] : rdx[k];
        out[c1].distance = d1;
        out[c1].parent = parent;
        out[c2].distance = d2;
        out[c2].parent = parent;
        out[parent].level = std::max(out[c1].level, out[c2].level) + 1;
        out[parent].child[0] = c1;
        out[parent].child[1] = c2;
    }
    return MSA_OK;
}

}  // namespace msa
