// All-pairs Needleman-Wunsch kernels for sm_100a.
//
// Recurrence (linear gap, global alignment), exactly the one of
// sequential::align_pair (src/pairwise/needleman/impl/sequential.cpp:29-68):
//   H[0][j] = -j*g, H[i][0] = -i*g,
//   H[i][j] = max(H[i-1][j-1] + T[a_i][b_j], H[i][j-1] - g, H[i-1][j] - g).
// Scores are small integers, so int32 (or, where a host-side bound proves it
// cannot overflow, 16-bit lanes) reproduces the reference's float scores
// exactly.
//
// Work layout: one warp runs one task. A task is one (rows, cols) pair, or on
// the 16-bit path two pairs sharing the column sequence (the two rows
// sequences of a rows pair, one per 16-bit half). Lane k owns R consecutive
// rows of a 32*R-row strip and sweeps the columns one step behind lane k-1:
// the cell above its first row arrives from lane k-1 by __shfl_up_sync, so a
// strip advances one anti-diagonal per step with no block-wide barrier. Strips
// of a long rows sequence are chained through a per-warp boundary row in
// global memory. Substitution scores come from a per-sequence score profile
// (one int8 row per residue code) staged per strip in shared memory, in planes
// whose 16-byte (or 8-byte) loads are bank-conflict free whatever codes the
// lanes hold; the batched kernel keeps part of each strip as packed bytes
// (Layout) to halve those rows' shared-memory traffic.
#include <cstdio>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "msa_internal.hpp"

namespace msa {
namespace dev {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kEnd = MSA_UNIT_END;

// Sign-extended byte K of w.
template <int K>
__device__ __forceinline__ int32_t sbyte(uint32_t w)
{
    int32_t r;
    asm("prmt.b32 %0, %1, 0, %2;" : "=r"(r) : "r"(w), "n"((K) | ((K | 8) << 4) | ((K | 8) << 8) | ((K | 8) << 12)));
    return r;
}

// Two sign-extended bytes K of lo and hi packed as int16x2 (lo in bits 0-15).
template <int K>
__device__ __forceinline__ uint32_t sbyte2(uint32_t lo, uint32_t hi)
{
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(lo), "r"(hi),
        "n"((K) | ((K | 8) << 4) | ((4 + K) << 8) | (((4 + K) | 8) << 12)));
    return r;
}

__device__ __forceinline__ uint32_t dup16(int32_t v) { return ((uint32_t) v & 0xffffu) | ((uint32_t) v << 16); }

// One cell: max(up - g, max(left - g, diag + s)). The inner max depends only on
// the previous column, so the serial chain down a lane's rows is one DPX op.
struct Wide {
    using W = int32_t;
    __device__ static __forceinline__ W cell(W d, W s, W left, W up, W ng)
    {
        const W ds = d + s;
        const W t = __viaddmax_s32(left, ng, ds);
        return __viaddmax_s32(up, ng, t);
    }
    __device__ static __forceinline__ W splat(int32_t v) { return v; }
    // max(left - g, diag + s): the part of a cell that needs only the previous column.
    __device__ static __forceinline__ W cell_part(W d, W s, W left, W ng) { return __viaddmax_s32(left, ng, d + s); }
    // max(up - g, part): the serial part down a lane's rows.
    __device__ static __forceinline__ W cell_chain(W up, W ng, W part) { return __viaddmax_s32(up, ng, part); }
};

// Two cells per 32-bit lane (16-bit halves: the two rows sequences of a rows
// pair). The lane state is not H but T(i,j) = H(i,j) + g*(i + j), unsigned per
// half. The gap terms cancel out of the recurrence:
//   T = max(T_left, T_up, T_diag + (s + 2g)),
// one vadd2 (FMA pipe, off the row chain) and one vimax3_u16x2 (ALU pipe, the
// only operation on the chain down a lane's rows); the staged profile words
// hold s + 2g. Row 0 and column 0 of T are 0. Over every path T = the sum of
// (s + 2g) over its matched cells, so 0 <= T(i,j) <= min(i,j)*(smax + 2g) when
// smin + 2g >= 0 (narrow_ok checks both), and the diagonal candidate never
// exceeds the cell it competes for: no half leaves [0, 0xffff]. Every operation
// stays inside its 16-bit half, so rows past a sequence's end (padding, or the
// shorter sequence of the pair) hold values that never reach a scored cell.
struct Narrow {
    using W = uint32_t;
    // H(rows, cols) from the low or high half of T(rows, cols).
    __device__ static __forceinline__ int32_t lo(W w, int32_t g, int rows, int cols) { return (int32_t) (w & 0xffffu) - g * (rows + cols); }
    __device__ static __forceinline__ int32_t hi(W w, int32_t g, int rows, int cols) { return (int32_t) (w >> 16) - g * (rows + cols); }
    __device__ static __forceinline__ W splat(int32_t v) { return dup16(v); }
};

// R profile bytes of one lane for residue code b, from the staged strip.
// Layout [code][plane][lane][16] with R/16 planes (R >= 16) or [code][lane][R].
template <int R>
struct ProfWords {
    static constexpr int NW = R / 4;
    uint32_t w[NW];
    __device__ __forceinline__ void load(const int8_t *sprof, int b, int lane)
    {
        constexpr int SH = 32 * R;
        if constexpr(R >= 16) {
#pragma unroll
            for(int p = 0; p < R / 16; ++p) {
                const uint4 v = *reinterpret_cast<const uint4 *>(sprof + b * SH + p * 512 + lane * 16);
                w[4 * p + 0] = v.x; w[4 * p + 1] = v.y; w[4 * p + 2] = v.z; w[4 * p + 3] = v.w;
            }
        } else if constexpr(R == 8) {
            const uint2 v = *reinterpret_cast<const uint2 *>(sprof + b * SH + lane * 8);
            w[0] = v.x; w[1] = v.y;
        } else {
            static_assert(R == 4, "R must be 4, 8, 16 or 32");
            w[0] = *reinterpret_cast<const uint32_t *>(sprof + b * SH + lane * 4);
        }
    }
};

// Copies strip rows [i0, i0 + 32R) of a sequence profile ([code][Lp] int8,
// global) into the warp's shared staging area.
template <int R>
__device__ __forceinline__ void stage_profile(int8_t *sprof, const int8_t *__restrict__ gprof,
                                              uint32_t lp, int i0, int lane)
{
    constexpr int SH = 32 * R;
    constexpr int CH = SH / 16;   // 16-byte chunks per code row
    for(int c = lane; c < kAlpha * CH; c += 32) {
        const int b = c / CH, w = c - b * CH;
        const uint4 v = __ldg(reinterpret_cast<const uint4 *>(gprof + (size_t) b * lp + i0) + w);
        int dst;
        if constexpr(R >= 16) {
            const int ln = w / (R / 16), pl = w - ln * (R / 16);
            dst = b * SH + pl * 512 + ln * 16;
        } else {
            dst = b * SH + w * 16;   // [code][lane][R] is the natural order for R <= 16
        }
        *reinterpret_cast<uint4 *>(sprof + dst) = v;
    }
}

// Runs one task in 32-bit lanes on the calling warp (the plain and the
// reference-orientation kernels): ncolsA columns of colsA against nrows rows.
// kSkip: END units in the columns copy the left neighbour
// (sequential.cpp:53-60) instead of scoring. Returns H[nrows][ncolsA] (resA);
// colsB, ncolsB and resB are unused (resB = 0).
template <int R, class K, bool kSkip>
__device__ __forceinline__ void run_task(const int8_t *__restrict__ gprof, uint32_t lp, int nrows,
                                         const uint8_t *__restrict__ colsA, int ncolsA,
                                         const uint8_t *__restrict__ colsB, int ncolsB,
                                         int8_t *sprof, uint32_t *__restrict__ bound,
                                         int32_t g, int lane, int32_t &resA, int32_t &resB)
{
    static_assert(std::is_same<K, Wide>::value, "run_task sweeps 32-bit lanes");
    using W = typename K::W;
    constexpr int SH = 32 * R;
    const int nstrips = (nrows + SH - 1) / SH;
    const W ng = K::splat(-g);
    int32_t outA = 0, outB = 0;

    for(int s = 0; s < nstrips; ++s) {
        const int i0 = s * SH;
        const bool first = (s == 0);
        const bool last = (s == nstrips - 1);
        const int rl = nrows - 1 - i0;              // last row's offset (meaningful in the last strip)
        const int klast = last ? rl / R : 31;
        const int rlast = rl - (rl / R) * R;

        __syncwarp();
        stage_profile<R>(sprof, gprof, lp, i0, lane);
        __syncwarp();

        W H[R];
#pragma unroll
        for(int r = 0; r < R; ++r) H[r] = K::splat(-(i0 + lane * R + r + 1) * g);
        W diag = K::splat(-(i0 + lane * R) * g);    // H[row_top - 1][0]
        W hlast = H[R - 1];

        // Boundary row of the previous strip, prefetched 32 columns at a time
        // (lane q holds column c0 + q); lane 0 picks its column by shuffle.
        uint32_t bq_cur = 0, bq_nxt = 0;
        if(!first) {
            bq_cur = bound[lane];
            bq_nxt = bound[32 + lane];
        }
        int clampA = ncolsA - 1;
        uint32_t curA = colsA[min(max(-lane, 0), clampA)];

        const int tend = ncolsA + klast;
        for(int t = 0; t < tend; ++t) {
            W up = __shfl_up_sync(kFull, hlast, 1);
            if(!first) {
                if((t & 31) == 0 && t > 0) {
                    bq_cur = bq_nxt;
                    bq_nxt = bound[t + 32 + lane];
                }
                const uint32_t bv = __shfl_sync(kFull, bq_cur, t & 31);
                if(lane == 0) up = (W) bv;
            } else if(lane == 0) {
                up = K::splat(-(t + 1) * g);
            }
            const int j = t - lane;
            const int jn = min(max(j + 1, 0), clampA);
            const uint32_t nxtA = colsA[jn];

            if(j >= 0 && j < ncolsA) {
                const bool skip = kSkip && curA == (uint32_t) kEnd;
                if(!skip) {
                    ProfWords<R> pa;
                    pa.load(sprof, (int) curA, lane);
                    W d = diag, u = up;
#pragma unroll
                    for(int q = 0; q < R / 4; ++q) {
#pragma unroll
                        for(int k = 0; k < 4; ++k) {
                            const int r = 4 * q + k;
                            W sc;
                            if(k == 0) sc = sbyte<0>(pa.w[q]);
                            else if(k == 1) sc = sbyte<1>(pa.w[q]);
                            else if(k == 2) sc = sbyte<2>(pa.w[q]);
                            else sc = sbyte<3>(pa.w[q]);
                            const W h = K::cell(d, sc, H[r], u, ng);
                            d = H[r];
                            H[r] = h;
                            u = h;
                        }
                    }
                }
                hlast = H[R - 1];
                if(!last && lane == 31) bound[j] = (uint32_t) hlast;
                if(last && lane == klast && j == ncolsA - 1) {
                    W v = H[0];
#pragma unroll
                    for(int r = 1; r < R; ++r) if(r == rlast) v = H[r];
                    outA = (int32_t) v;
                }
                diag = up;
            }
            curA = nxtA;
        }
        if(last) {
            resA = __shfl_sync(kFull, outA, klast);
            resB = __shfl_sync(kFull, outB, klast);
        }
    }
    __syncwarp();
}

__device__ __forceinline__ uint64_t tri_index(uint32_t i, uint32_t j)
{
    const uint64_t hi = i > j ? i : j, lo = i > j ? j : i;
    return hi * (hi - 1) / 2 + lo;
}

}  // namespace dev

// ---------------------------------------------------------------- params

struct NwParams {
    const uint8_t *units;
    const uint64_t *uoff;
    const uint32_t *eff;
    const uint32_t *plen;
    const int8_t *prof;
    const uint64_t *poff;
    const uint32_t *plp;
    const uint32_t *sorted;     // clean sequences, eff descending
    uint32_t nclean;
    const uint64_t *row_task;   // persistent: first task of each sorted row (nclean + 1)
    const uint8_t *row_narrow;  // persistent: 16-bit tasks for this row
    uint64_t ntasks;
    const uint32_t *gpairs;     // generic path: (rows orig, cols orig) pairs
    uint64_t ngeneric;
    uint32_t *bound;            // per resident warp: bound_stride words
    uint64_t bound_stride;
    int32_t *out;
    int32_t g;
    unsigned long long *counter;
};

// Sorted-space pair (a, b), a < b, from its a-major linear index k.
__device__ __forceinline__ void decode_pair(uint64_t k, uint32_t n, uint32_t &a, uint32_t &b)
{
    // Row a starts at a*(2n - a - 1)/2.
    const double nn = (double) n - 0.5;
    double x = nn - sqrt(nn * nn - 2.0 * (double) k);
    int64_t aa = (int64_t) floor(x);
    if(aa < 0) aa = 0;
    auto start = [n](int64_t r) -> uint64_t { return (uint64_t) r * (2 * (uint64_t) n - (uint64_t) r - 1) / 2; };
    while(aa > 0 && start(aa) > k) --aa;
    while(start(aa + 1) <= k) ++aa;
    a = (uint32_t) aa;
    b = (uint32_t) (aa + 1 + (k - start(aa)));
}

template <int R>
__device__ __forceinline__ void clean_pair_task(const NwParams &p, uint32_t a, uint32_t b,
                                                int8_t *sprof, uint32_t *bound, int lane)
{
    const uint32_t ri = p.sorted[a], ci = p.sorted[b];
    int32_t ra = 0, rb = 0;
    dev::run_task<R, dev::Wide, false>(p.prof + p.poff[ri], p.plp[ri], (int) p.eff[ri],
                                       p.units + p.uoff[ci], (int) p.eff[ci], nullptr, 0,
                                       sprof, bound, p.g, lane, ra, rb);
    if(lane == 0) p.out[dev::tri_index(ri, ci)] = ra;
}

// Plain: one launch per length bucket (a range of the a-major pair order),
// each warp takes pairs k_lo + w, k_lo + w + W, ... in a fixed stride.
template <int R, int WPB>
__global__ void __launch_bounds__(WPB * 32) nw_plain_kernel(NwParams p, uint64_t k_lo, uint64_t k_hi)
{
    extern __shared__ __align__(16) int8_t smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int8_t *sprof = smem + warp * (kAlpha * 32 * R);
    const uint64_t gw = (uint64_t) blockIdx.x * WPB + warp;
    const uint64_t nw = (uint64_t) gridDim.x * WPB;
    uint32_t *bound = p.bound + gw * p.bound_stride;
    for(uint64_t k = k_lo + gw; k < k_hi; k += nw) {
        uint32_t a, b;
        decode_pair(k, p.nclean, a, b);
        clean_pair_task<R>(p, a, b, sprof, bound, lane);
    }
}

// ---------------------------------------------------------------- batched kernel
//
// One persistent launch over every clean pair. The length-sorted sequences
// are taken two at a time as a rows pair (X1, X2) = (sorted 2k, sorted 2k+1);
// a task is one rows pair against a group of W consecutive column sequences,
// one per warp of the CTA. On the 16-bit path the two rows sequences share
// every 32-bit lane: X1 in the low half, X2 in the high half, against the same
// column residue, so one staged profile word is already the packed score pair
// and each lane does two cells per instruction. The profile strip is staged
// once per CTA and shared by its W warps. Where the 16-bit bound fails the
// task runs both rows sequences one after the other in 32-bit lanes.
// CTAs take tasks from a global counter in cost order (longest rows pairs
// first), so the tail of the launch is the cheapest work.

// One all-pairs job as the batched kernels see it: its store, score profiles,
// length order, per-rows-pair 16-bit flags and output triangle.
struct JobView {
    const uint8_t *units;
    const uint64_t *uoff;
    const uint32_t *eff;
    const int8_t *prof;
    const uint64_t *poff;
    const uint32_t *plp;
    const uint32_t *sorted;     // clean sequences, eff descending
    const uint8_t *row_narrow;  // per rows pair k: kRowNarrow, and kRowQuad for the first of a stacked pair
    int32_t *out;
    uint32_t nclean;
    int32_t g;
};

// row_narrow flags: 16-bit lanes; rows pairs k and k + 1 stacked in one warp
// (quad_task), their tasks all under k.
constexpr uint8_t kRowNarrow = 1, kRowQuad = 2;

struct BatchParams {
    JobView job;
    uint32_t npairs_rows;       // number of rows pairs, ceil(nclean / 2)
    const uint64_t *row_task;   // first task of each rows pair (npairs_rows + 1)
    uint64_t ntasks;            // tasks of this launch: task_base .. task_base + ntasks - 1
    uint64_t task_base;
    uint32_t gchunk;            // column groups per task of a single-strip rows pair
    uint32_t *bound;
    uint64_t bound_stride;
    unsigned long long *counter;
};

// Merged launches of the serving loop: explicit (job slot, rows pair, column
// group) tasks over several jobs.
struct ServeParams {
    const JobView *jobs;
    const uint4 *tasks;
    uint64_t ntasks;
    uint32_t *bound;
    uint64_t bound_stride;
    unsigned long long *counter;
};

namespace dev {

// Shared-memory layout of one strip's profile for R rows per lane, per code:
// R16 rows as 32-bit words in planes [lane][4 words] of 4 rows (one 16-byte
// load per lane and plane, bank-conflict free whatever codes the lanes hold),
// then a half plane [lane][2 words] when R16 is 2 mod 4; then, on 16-bit lanes,
// R8 rows as packed bytes, one word holding rows r and r + 1 of both sequences,
// in planes [lane][4 words] of 8 rows and a half plane [lane][2 words] of 4
// rows when R8 is 4 mod 8. A packed row costs one PRMT (ALU pipe) and half the
// shared-memory bytes of a 16-bit row. R8 = 8 floor(R/16) (a third to a half of
// a long strip's rows) balances the shared-memory data pipe, the bound of
// 16-bit rows alone, against the ALU pipe and issue: on c3 it measured 16.07
// TCUPS against 14.81 with no packed rows and 15.96 with R8 = 4 floor(R/8).
template <int R, bool kNarrow, bool kPack = true> struct Layout {
    static constexpr int R8 = kNarrow && kPack ? 8 * (R / 16) : 0;
    static constexpr int R16 = R - R8;
    static constexpr int P16 = R16 / 4;                      // full 16-bit planes
    static constexpr bool kHalf = R16 % 4 != 0;
    static constexpr int HALF = P16 * 128;                   // word offset of the 16-bit half plane
    static constexpr int PACK = HALF + (kHalf ? 64 : 0);     // word offset of the packed planes
    static constexpr int P8 = R8 / 8;                        // full packed planes
    static constexpr int PHALF = PACK + P8 * 128;            // word offset of the packed half plane
    static constexpr int SH = PHALF + (R8 % 8 ? 64 : 0);     // words per code
};

// PRMT of w with a zero second operand.
template <int SEL>
__device__ __forceinline__ uint32_t prmt0(uint32_t w)
{
    uint32_t r;
    asm("prmt.b32 %0, %1, 0, %2;" : "=r"(r) : "r"(w), "n"(SEL));
    return r;
}

// Stages strip rows [i0, i0 + 32R) of the profile in shared memory (Layout).
// Narrow: word = (s(X1_i, b) + 2g, s(X2_i, b) + 2g) as 16x2 (see Narrow), or
// bytes (s1_i, s1_i+1, s2_i, s2_i+1) + 2g in the packed planes; rows of X2 past
// its profile (lp2) score 0. Wide: word = s(X1_i, b) as int32.
// The profile is read in 16-byte chunks (16 rows of one code), each thread
// issuing the loads of up to kStageBatch chunks before it converts and stores
// any, so one staging costs about one L2 round trip instead of one per chunk.
// Profile rows are 16-byte aligned: the per-sequence pitch is a multiple of
// 1024 and i0 a multiple of 64; lp2 is a multiple of 1024, so a chunk lies
// wholly inside or wholly past X2's profile.
constexpr int kStageBatch = 4;

// With msplit < 2R (16-bit lanes only), chunks m >= msplit (strip rows
// 16 msplit and on) come from a second rows pair, (g1b, g2b) at their row
// 16 (m - msplit): the stacked strip of quad_task.
template <int R, bool kNarrow, bool kPack = true>
__device__ __forceinline__ void stage_words(uint32_t *sprof, const int8_t *__restrict__ g1, uint32_t lp1,
                                            const int8_t *__restrict__ g2, uint32_t lp2, int i0, int32_t gap = 0,
                                            const int8_t *__restrict__ g1b = nullptr, uint32_t lp1b = 0,
                                            const int8_t *__restrict__ g2b = nullptr, uint32_t lp2b = 0,
                                            int msplit = 1 << 30)
{
    using L = Layout<R, kNarrow, kPack>;
    constexpr int SH = L::SH;
    constexpr int CH = 2 * R;                 // 16-byte chunks per code row (32R rows)
    constexpr int TOTAL = kAlpha * CH;
    const int nt = blockDim.x;
    if constexpr(kNarrow) {
        static_assert(R % 2 == 0, "16-bit lanes take an even number of rows");
        const uint32_t gg = ((uint32_t) (2 * gap) & 0xffffu) * 0x10001u;
        for(int c0 = threadIdx.x; c0 < TOTAL; c0 += kStageBatch * nt) {
            uint4 va[kStageBatch], vb[kStageBatch];
#pragma unroll
            for(int u = 0; u < kStageBatch; ++u) {
                const int c = c0 + u * nt;
                va[u] = vb[u] = make_uint4(0, 0, 0, 0);
                if(c < TOTAL) {
                    const int b = c / CH, m = c - b * CH;
                    if(m < msplit) {
                        va[u] = __ldg(reinterpret_cast<const uint4 *>(g1 + (size_t) b * lp1 + i0) + m);
                        if((uint32_t) (i0 + 16 * m) < lp2)
                            vb[u] = __ldg(reinterpret_cast<const uint4 *>(g2 + (size_t) b * lp2 + i0) + m);
                    } else {
                        const int mb = m - msplit;
                        va[u] = __ldg(reinterpret_cast<const uint4 *>(g1b + (size_t) b * lp1b) + mb);
                        if((uint32_t) (16 * mb) < lp2b)
                            vb[u] = __ldg(reinterpret_cast<const uint4 *>(g2b + (size_t) b * lp2b) + mb);
                    }
                }
            }
#pragma unroll
            for(int u = 0; u < kStageBatch; ++u) {
                const int c = c0 + u * nt;
                if(c >= TOTAL) break;
                const int b = c / CH, m = c - b * CH;
                uint32_t *code = sprof + b * SH;
                const uint32_t wa[4] = {va[u].x, va[u].y, va[u].z, va[u].w};
                const uint32_t wb[4] = {vb[u].x, vb[u].y, vb[u].z, vb[u].w};
#pragma unroll
                for(int k = 0; k < 8; ++k) {   // two-row group k: rows 16m + 2k, 16m + 2k + 1
                    uint2 o;
                    if(k & 1) {
                        o.x = __vadd2(sbyte2<2>(wa[k >> 1], wb[k >> 1]), gg);
                        o.y = __vadd2(sbyte2<3>(wa[k >> 1], wb[k >> 1]), gg);
                    } else {
                        o.x = __vadd2(sbyte2<0>(wa[k >> 1], wb[k >> 1]), gg);
                        o.y = __vadd2(sbyte2<1>(wa[k >> 1], wb[k >> 1]), gg);
                    }
                    const int row = 16 * m + 2 * k, ln = row / R, r = row - ln * R;
                    if(r < 4 * L::P16) {
                        *reinterpret_cast<uint2 *>(code + (r >> 2) * 128 + ln * 4 + (r & 3)) = o;
                    } else if(r < L::R16) {
                        *reinterpret_cast<uint2 *>(code + L::HALF + ln * 2) = o;
                    } else {
                        const int wi = (r - L::R16) >> 1;   // packed word of rows r, r + 1
                        uint32_t pk;
                        asm("prmt.b32 %0, %1, %2, 0x6240;" : "=r"(pk) : "r"(o.x), "r"(o.y));
                        if(wi < 4 * L::P8) code[L::PACK + (wi >> 2) * 128 + ln * 4 + (wi & 3)] = pk;
                        else code[L::PHALF + ln * 2 + (wi - 4 * L::P8)] = pk;
                    }
                }
            }
        }
    } else {
        static_assert(R % 4 == 0, "32-bit lanes use full planes");
        constexpr int PL = R / 4;        // planes per lane
        for(int c0 = threadIdx.x; c0 < TOTAL; c0 += kStageBatch * nt) {
            uint4 va[kStageBatch];
#pragma unroll
            for(int u = 0; u < kStageBatch; ++u) {
                const int c = c0 + u * nt;
                va[u] = make_uint4(0, 0, 0, 0);
                if(c < TOTAL) {
                    const int b = c / CH, m = c - b * CH;
                    va[u] = __ldg(reinterpret_cast<const uint4 *>(g1 + (size_t) b * lp1 + i0) + m);
                }
            }
#pragma unroll
            for(int u = 0; u < kStageBatch; ++u) {
                const int c = c0 + u * nt;
                if(c >= TOTAL) break;
                const int b = c / CH, m = c - b * CH;
                const uint32_t wa[4] = {va[u].x, va[u].y, va[u].z, va[u].w};
#pragma unroll
                for(int k = 0; k < 4; ++k) {   // 4-row group 4m + k
                    const int rg = 4 * m + k, ln = rg / PL, pl = rg - ln * PL;
                    uint4 o;
                    o.x = (uint32_t) sbyte<0>(wa[k]);
                    o.y = (uint32_t) sbyte<1>(wa[k]);
                    o.z = (uint32_t) sbyte<2>(wa[k]);
                    o.w = (uint32_t) sbyte<3>(wa[k]);
                    *reinterpret_cast<uint4 *>(sprof + b * SH + pl * 128 + ln * 4) = o;
                }
            }
        }
    }
}

template <bool V> struct Guard { static constexpr bool value = V; };

// Where the row above a strip comes from (sweep_strip's kTop):
//   kTopBound  the boundary row in `bound` (any strip; the last row is stored
//              back when store_bound);
//   kTopZero   row zero of the gap-free state, 0, above lane 0 (a strip that
//              is the first and the last one, 16-bit lanes only);
//   kTopStack  as kTopZero, and lanes 16..31 hold a second rows pair of its
//              own whose row zero sits above lane 16 (see quad_task).
constexpr int kTopBound = 0, kTopZero = 1, kTopStack = 2;

// Sweeps one strip (rows [i0, i0 + 32R)) of one column sequence on the calling
// warp. `bound` holds the row above the strip on entry (column j at index j)
// and, when store_bound, the strip's last row on exit. After the call, lane k's
// H registers hold the strip's rows at the last column it reached
// (tend - 1 - lane). Steps run in groups of 8 (the loop bookkeeping of a group
// is shared by 8 columns); only the fill and drain groups, where some lanes
// sit outside [0, ncols), test the lane's column.
template <int R, class K, bool kPack = true, int kTop = kTopBound>
__device__ __forceinline__ void sweep_strip(const uint32_t *__restrict__ sprof, const uint8_t *__restrict__ cols,
                                            int ncols, uint32_t *__restrict__ bound, int i0, int tend,
                                            bool store_bound, int32_t g, int lane, typename K::W (&H)[R])
{
    using W = typename K::W;
    constexpr bool kB = std::is_same<K, Narrow>::value;
    using L = Layout<R, kB, kPack>;
    constexpr int SH = L::SH;
    const W ng = K::splat(-g);
    W diag;
    if constexpr(kB) {
#pragma unroll
        for(int r = 0; r < R; ++r) H[r] = 0u;   // column 0 of T
        diag = 0u;
    } else {
#pragma unroll
        for(int r = 0; r < R; ++r) H[r] = K::splat(-(i0 + lane * R + r + 1) * g);
        diag = K::splat(-(i0 + lane * R) * g);
    }
    W hlast = H[R - 1];
    static_assert(kTop == kTopBound || kB, "row zero is 0 only in the gap-free 16-bit state");
    uint32_t bq_cur = 0, bq_nxt = 0;
    if constexpr(kTop == kTopBound) {
        bq_cur = bound[lane];
        bq_nxt = bound[32 + lane];
    }
    const uint32_t *prow = sprof + lane * 4;
    const int half_off = L::HALF - lane * 2;      // the 16-bit half plane, from prow
    const int phalf_off = L::PHALF - lane * 2;    // the packed half plane, from prow
    const bool st31 = store_bound && lane == 31;
    int j = -lane;
    uint32_t cur = cols[j], nxt = cols[j + 1];   // columns -32..ncols+35 lie in the padded store

    auto group = [&](int t0, auto guard) {
        constexpr bool kG = decltype(guard)::value;
        if(kTop == kTopBound && (t0 & 31) == 0 && t0 > 0) {
            bq_cur = bq_nxt;
            bq_nxt = bound[t0 + 32 + lane];
        }
#pragma unroll
        for(int u = 0; u < 8; ++u) {
            W up = __shfl_up_sync(kFull, hlast, 1);
            if constexpr(kTop == kTopBound) {
                const uint32_t bv = __shfl_sync(kFull, bq_cur, (t0 & 31) + u);
                if(lane == 0) up = (W) bv;
            } else if constexpr(kTop == kTopZero) {
                if(lane == 0) up = 0u;
            } else {
                if((lane & 15) == 0) up = 0u;
            }
            if(!kG || (unsigned) j < (unsigned) ncols) {
                const uint32_t *pb = prow + cur * SH;
                W sc[4];
                auto load_plane = [&](int q) {   // 16-bit plane q (q == P16: the half plane)
                    if(q < L::P16) {
                        const uint4 v = *reinterpret_cast<const uint4 *>(pb + q * 128);
                        sc[0] = (W) v.x; sc[1] = (W) v.y; sc[2] = (W) v.z; sc[3] = (W) v.w;
                    } else {
                        const uint2 v = *reinterpret_cast<const uint2 *>(pb + half_off);
                        sc[0] = (W) v.x; sc[1] = (W) v.y;
                    }
                };
                load_plane(0);
                if constexpr(kB) {
                    // T = max(T_left, T_up, T_diag + s + 2g); see Narrow.
                    W above = up, dprev = diag;
                    uint4 pk;
#pragma unroll
                    for(int r = 0; r < R; ++r) {
                        W sr;
                        if(r < L::R16) {
                            if(r > 0 && (r & 3) == 0) load_plane(r >> 2);
                            sr = sc[r & 3];
                        } else {
                            const int rr = r - L::R16;
                            if((rr & 7) == 0) {
                                if((rr >> 3) < L::P8) {
                                    pk = *reinterpret_cast<const uint4 *>(pb + L::PACK + (rr >> 3) * 128);
                                } else {
                                    const uint2 v = *reinterpret_cast<const uint2 *>(pb + phalf_off);
                                    pk.x = v.x;
                                    pk.y = v.y;
                                }
                            }
                            const int wi = (rr >> 1) & 3;
                            const uint32_t w = wi == 0 ? pk.x : wi == 1 ? pk.y : wi == 2 ? pk.z : pk.w;
                            sr = (rr & 1) ? prmt0<0x4341>(w) : prmt0<0x4240>(w);
                        }
                        const W D = __vadd2(dprev, sr);
                        dprev = H[r];
                        H[r] = __vimax3_u16x2(H[r], above, D);
                        above = H[r];
                    }
                } else {
                static_assert(R % 4 == 0, "32-bit lanes use full planes");
                // Row r needs the old H[r-1] (diagonal) and old H[r] (left): the
                // off-chain part for row r+1 is computed before row r is
                // overwritten, so no register copies are needed.
                W pn = K::cell_part(diag, sc[0], H[0], ng);
                W u_ = up;
#pragma unroll
                for(int r = 0; r < R; ++r) {
                    const W pr = pn;
                    if(r + 1 < R) {
                        if(((r + 1) & 3) == 0) load_plane((r + 1) >> 2);
                        pn = K::cell_part(H[r], sc[(r + 1) & 3], H[r + 1], ng);
                    }
                    H[r] = K::cell_chain(u_, ng, pr);
                    u_ = H[r];
                }
                }
                hlast = H[R - 1];
                if constexpr(kTop == kTopBound)
                    if(st31) bound[j] = (uint32_t) hlast;
                diag = up;
            }
            cur = nxt;
            nxt = cols[j + 2];
            ++j;
        }
    };

    const int tend4 = (tend + 7) & ~7;
    int t0 = 0;
#pragma unroll 1
    for(; t0 < tend4 && t0 < 32; t0 += 8) group(t0, Guard<true>{});
#pragma unroll 1
    for(; t0 + 7 < ncols; t0 += 8) group(t0, Guard<false>{});   // every lane inside [0, ncols)
#pragma unroll 1
    for(; t0 < tend4; t0 += 8) group(t0, Guard<true>{});
}

template <int R, class K>
__device__ __forceinline__ typename K::W pick_row(const typename K::W (&H)[R], int r)
{
    typename K::W v = H[0];
#pragma unroll
    for(int q = 1; q < R; ++q) if(q == r) v = H[q];
    return v;
}

// The column sequences of one task: sorted b0, b0 + bstep, ... (ngrp of them
// for this warp), each against the rows pair (x1, x2) of a job.
struct TaskCols {
    const JobView *jv;
    uint32_t x1, x2, a2;   // rows sequences (original index) and x2's sorted index
    uint32_t b0, bstep, ngrp;
};

// One task's work for a 16-bit rows pair with strips of 32R rows. With a
// single strip (nst == 1) the strip is staged once and swept against every
// column sequence of the task; otherwise the task has one column sequence per
// warp and every strip is staged in turn. Only the first staging of a
// single-strip task and the stagings of a multi-strip task synchronise the
// CTA, so the loop counts and nst are CTA-uniform.
template <int R, bool kPack>
__device__ __noinline__ void narrow_task(uint32_t *sprof, const int8_t *g1, uint32_t lp1, const int8_t *g2,
                                         uint32_t lp2, int e1, int e2, int nst, const TaskCols &tc, uint32_t *bound,
                                         int32_t g, int lane)
{
    constexpr int SH = 32 * R;
    const JobView &jv = *tc.jv;
    const int s2 = (e2 - 1) / SH;
    for(uint32_t t = 0; t < tc.ngrp; ++t) {
        const uint32_t b = tc.b0 + t * tc.bstep;
        const bool has = b < jv.nclean;
        const uint32_t y = has ? jv.sorted[b] : tc.x1;
        const int ncols = has ? (int) jv.eff[y] : 0;
        const uint8_t *cols = jv.units + jv.uoff[y];
        // Row zero of the DP (0 in the T state) as the boundary above the
        // first of several strips (a single strip takes it as a constant).
        if(has && nst > 1) for(int jj = lane; jj < ncols + 96; jj += 32) bound[jj] = 0u;
        int32_t r1 = 0, r2 = 0;
        for(int s = 0; s < nst; ++s) {
            const int i0 = s * SH;
            if(t == 0 || nst > 1) {
                __syncthreads();
                stage_words<R, true, kPack>(sprof, g1, lp1, g2, lp2, i0, g);
                __syncthreads();
            }
            if(has) {
                const bool last = s == nst - 1;
                const int k1 = last ? (e1 - 1 - i0) / R : 31;
                Narrow::W H[R];
                __syncwarp();
                if(nst == 1)
                    sweep_strip<R, Narrow, kPack, kTopZero>(sprof, cols, ncols, bound, i0, ncols + k1, false, g, lane, H);
                else
                    sweep_strip<R, Narrow, kPack>(sprof, cols, ncols, bound, i0, ncols + k1, !last, g, lane, H);
                __syncwarp();
                if(s == s2) {
                    const int rr = e2 - 1 - i0;
                    r2 = __shfl_sync(kFull, Narrow::hi(pick_row<R, Narrow>(H, rr % R), g, e2, ncols), rr / R);
                }
                if(last) {
                    const int rr = e1 - 1 - i0;
                    r1 = __shfl_sync(kFull, Narrow::lo(pick_row<R, Narrow>(H, rr % R), g, e1, ncols), rr / R);
                }
            }
        }
        if(has && lane == 0) {
            jv.out[tri_index(tc.x1, y)] = r1;
            if(b != tc.a2) jv.out[tri_index(tc.x2, y)] = r2;
        }
    }
}

// One rows sequence (x1 when h == 0, x2 when h == 1) in 32-bit lanes with
// strips of 32R rows, against the task's column sequences; staging as in
// narrow_task.
template <int R>
__device__ __noinline__ void wide_task(uint32_t *sprof, const int8_t *g1, uint32_t lp1, int e1, int nst, int h,
                                       const TaskCols &tc, uint32_t *bound, int32_t g, int lane)
{
    constexpr int SH = 32 * R;
    const JobView &jv = *tc.jv;
    const uint32_t xr = h ? tc.x2 : tc.x1;
    for(uint32_t t = 0; t < tc.ngrp; ++t) {
        const uint32_t b = tc.b0 + t * tc.bstep;
        const bool mine = b < jv.nclean && !(h == 1 && b == tc.a2);
        const uint32_t y = mine ? jv.sorted[b] : xr;
        const int ncols = mine ? (int) jv.eff[y] : 0;
        const uint8_t *cols = jv.units + jv.uoff[y];
        if(mine) for(int jj = lane; jj < ncols + 96; jj += 32) bound[jj] = (uint32_t) (-(jj + 1) * g);
        int32_t res = 0;
        for(int s = 0; s < nst; ++s) {
            const int i0 = s * SH;
            if(t == 0 || nst > 1) {
                __syncthreads();
                stage_words<R, false>(sprof, g1, lp1, nullptr, 0, i0);
                __syncthreads();
            }
            if(mine) {
                const bool last = s == nst - 1;
                const int k1 = last ? (e1 - 1 - i0) / R : 31;
                Wide::W H[R];
                __syncwarp();
                sweep_strip<R, Wide>(sprof, cols, ncols, bound, i0, ncols + k1, !last, g, lane, H);
                __syncwarp();
                if(last) {
                    const int rr = e1 - 1 - i0;
                    res = __shfl_sync(kFull, pick_row<R, Wide>(H, rr % R), rr / R);
                }
            }
        }
        if(mine && lane == 0) jv.out[tri_index(xr, y)] = res;
    }
}

// Two short rows pairs in one warp: pair A (sorted 2k, 2k+1) on lanes 0..15
// and pair B (sorted 2k+2, 2k+3) on lanes 16..31, R rows per lane, so each
// pair has 16R >= its rows in one strip; both sweep the same column
// sequences (those of pair A: sorted 2k+1 + q W + warp). In the gap-free
// state row zero is 0, so lane 16 takes 0 from above instead of lane 15's
// last row, and the two halves never mix. A column is scored for a rows
// sequence only when it comes after it in the sorted order. Halves the
// per-step overhead per cell against a 16R-row strip on 32 lanes.
template <int R, bool kPack>
__device__ __noinline__ void quad_task(uint32_t *sprof, const JobView &jv, uint32_t k, uint32_t b0, uint32_t bstep,
                                       uint32_t ngrp, int32_t g, int lane)
{
    const uint32_t xa1 = jv.sorted[2 * k], xa2 = jv.sorted[2 * k + 1];
    const uint32_t xb1 = jv.sorted[2 * k + 2], xb2 = jv.sorted[2 * k + 3];
    const int ea1 = (int) jv.eff[xa1], ea2 = (int) jv.eff[xa2], eb1 = (int) jv.eff[xb1], eb2 = (int) jv.eff[xb2];
    for(uint32_t t = 0; t < ngrp; ++t) {
        const uint32_t b = b0 + t * bstep;
        const bool has = b < jv.nclean;
        const uint32_t y = has ? jv.sorted[b] : xa1;
        const int ncols = has ? (int) jv.eff[y] : 0;
        const uint8_t *cols = jv.units + jv.uoff[y];
        if(t == 0) {
            __syncthreads();
            stage_words<R, true, kPack>(sprof, jv.prof + jv.poff[xa1], jv.plp[xa1], jv.prof + jv.poff[xa2],
                                        jv.plp[xa2], 0, g, jv.prof + jv.poff[xb1], jv.plp[xb1],
                                        jv.prof + jv.poff[xb2], jv.plp[xb2], R);
            __syncthreads();
        }
        if(has) {
            Narrow::W H[R];
            __syncwarp();
            // Lane 31 is the last one to reach a column (pair B's rows).
            sweep_strip<R, Narrow, kPack, kTopStack>(sprof, cols, ncols, nullptr, 0, ncols + 31, false, g, lane, H);
            __syncwarp();
            auto take = [&](int rows, int lane0, bool hi) {
                const int rr = rows - 1;
                const Narrow::W w = pick_row<R, Narrow>(H, rr % R);
                const int32_t v = hi ? Narrow::hi(w, g, rows, ncols) : Narrow::lo(w, g, rows, ncols);
                return __shfl_sync(kFull, v, lane0 + rr / R);
            };
            const int32_t ra1 = take(ea1, 0, false), ra2 = take(ea2, 0, true);
            const int32_t rb1 = take(eb1, 16, false), rb2 = take(eb2, 16, true);
            if(lane == 0) {
                jv.out[tri_index(xa1, y)] = ra1;
                if(b > 2 * k + 1) jv.out[tri_index(xa2, y)] = ra2;
                if(b > 2 * k + 2) jv.out[tri_index(xb1, y)] = rb1;
                if(b > 2 * k + 3) jv.out[tri_index(xb2, y)] = rb2;
            }
        }
    }
}

// Strip plan for `rows` rows with at most 32*RMAX rows per strip: the fewest
// strips, each of 32R rows with R the smallest even number that covers them.
template <int RMAX>
__device__ __forceinline__ void strip_plan(int rows, int &nst, int &R)
{
    nst = (rows + 32 * RMAX - 1) / (32 * RMAX);
    R = (rows + 32 * nst - 1) / (32 * nst);
    R = (R + 1) & ~1;
}

}  // namespace dev

// Resident CTAs per SM the batched kernel is compiled for (register budget).
template <int RMAX, int W> struct BatchOcc { static constexpr int value = (RMAX == 32 ? 16 : 24) / W; };

// Column groups of W per task for rows pair k of a job with nclean clean
// sequences: `chunk` groups when its rows fit one strip of 32 RMAX rows (the
// strip is then staged once for all of them), else one. The host's task
// tables use the same rule.
__host__ __device__ __forceinline__ uint32_t groups_per_task(uint32_t e1, int rmax, uint32_t chunk)
{
    return e1 <= (uint32_t) (32 * rmax) ? chunk : 1u;
}

// One task: rows pair k (sorted 2k, 2k+1) of job `jv` against `ngrp` column
// groups starting at `grp` (group q: sorted 2k+1 + q*W + warp for each warp).
// All threads of the CTA call it.
template <int RMAX, int W, bool kPack>
__device__ __forceinline__ void rows_pair_task(const JobView &jv, uint32_t k, uint32_t grp, uint32_t ngrp,
                                               uint32_t *sprof_b, uint32_t *bound, int warp, int lane)
{
    const uint32_t a1 = 2 * k, a2 = min(2 * k + 1, jv.nclean - 1);
    const uint32_t x1 = jv.sorted[a1], x2 = jv.sorted[a2];
    const int e1 = (int) jv.eff[x1], e2 = (int) jv.eff[x2];
    dev::TaskCols tc{&jv, x1, x2, a2, 2 * k + 1 + grp * W + warp, (uint32_t) W, ngrp};

    if constexpr(RMAX == 32) {
        if(jv.row_narrow[k] & kRowQuad) {
            // Rows pairs k and k + 1 stacked (quad_task): R rows per lane, 16R
            // covering pair k's longer first sequence.
            int R = (e1 + 15) / 16;
            R = (R + 1) & ~1;
#define MSA_QUAD(RR) case RR: dev::quad_task<RR, kPack>(sprof_b, jv, k, tc.b0, tc.bstep, ngrp, jv.g, lane); break;
            switch(R) {
                MSA_QUAD(2) MSA_QUAD(4) MSA_QUAD(6) MSA_QUAD(8) MSA_QUAD(10) MSA_QUAD(12) MSA_QUAD(14) MSA_QUAD(16)
                MSA_QUAD(18) MSA_QUAD(20) MSA_QUAD(22) MSA_QUAD(24) MSA_QUAD(26) MSA_QUAD(28) MSA_QUAD(30)
                MSA_QUAD(32) default: break;
            }
#undef MSA_QUAD
            return;
        }
    }
    if(jv.row_narrow[k]) {
        int nst, R;
        dev::strip_plan<RMAX>(e1, nst, R);
        const int8_t *g1 = jv.prof + jv.poff[x1], *g2 = jv.prof + jv.poff[x2];
        const uint32_t lp1 = jv.plp[x1], lp2 = jv.plp[x2];
#define MSA_NARROW(RR) case RR: dev::narrow_task<RR, kPack>(sprof_b, g1, lp1, g2, lp2, e1, e2, nst, tc, bound, jv.g, lane); break;
        switch(R) {
            MSA_NARROW(2) MSA_NARROW(4) MSA_NARROW(6) MSA_NARROW(8) MSA_NARROW(10) MSA_NARROW(12) MSA_NARROW(14)
            MSA_NARROW(16)
            default:
                if constexpr(RMAX > 16) {
                    switch(R) {
                        MSA_NARROW(18) MSA_NARROW(20) MSA_NARROW(22) MSA_NARROW(24) MSA_NARROW(26) MSA_NARROW(28)
                        MSA_NARROW(30) MSA_NARROW(32) default: break;
                    }
                }
                break;
        }
#undef MSA_NARROW
    } else {
        for(int h = 0; h < 2; ++h) {
            if(h == 1 && a2 == a1) break;   // CTA-uniform
            const uint32_t xr = h ? x2 : x1;
            const int er = h ? e2 : e1;
            const int nst = (er + 32 * RMAX - 1) / (32 * RMAX);
            dev::wide_task<RMAX>(sprof_b, jv.prof + jv.poff[xr], jv.plp[xr], er, nst, h, tc, bound, jv.g, lane);
        }
    }
}

// kPack = false stages every profile row as 16-bit words (no packed-byte
// rows); it exists to measure what the packed rows contribute.
template <int RMAX, int W, bool kPack = true>
__global__ void __launch_bounds__(W * 32, BatchOcc<RMAX, W>::value) nw_batched_kernel(BatchParams p)
{
    extern __shared__ __align__(16) uint32_t sprof_b[];
    __shared__ unsigned long long task_q;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t *bound = p.bound + ((uint64_t) blockIdx.x * W + warp) * p.bound_stride;

    for(;;) {
        __syncthreads();
        if(threadIdx.x == 0) task_q = atomicAdd(p.counter, 1ull);
        __syncthreads();
        if(task_q >= p.ntasks) break;
        const unsigned long long q = task_q + p.task_base;
        uint32_t lo = 0, hi = p.npairs_rows - 1;
        while(lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if(p.row_task[mid] <= q) lo = mid; else hi = mid - 1;
        }
        const uint32_t groups = (p.job.nclean - 2 * lo - 1 + W - 1) / W;
        const uint32_t chunk = groups_per_task(p.job.eff[p.job.sorted[2 * lo]], RMAX, p.gchunk);
        const uint32_t grp = (uint32_t) (q - p.row_task[lo]) * chunk;
        rows_pair_task<RMAX, W, kPack>(p.job, lo, grp, min(chunk, groups - grp), sprof_b, bound, warp, lane);
    }
}

template <int RMAX, int W>
__global__ void __launch_bounds__(W * 32, BatchOcc<RMAX, W>::value) nw_serve_kernel(ServeParams p)
{
    extern __shared__ __align__(16) uint32_t sprof_b[];
    __shared__ unsigned long long task_q;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t *bound = p.bound + ((uint64_t) blockIdx.x * W + warp) * p.bound_stride;

    for(;;) {
        __syncthreads();
        if(threadIdx.x == 0) task_q = atomicAdd(p.counter, 1ull);
        __syncthreads();
        const unsigned long long q = task_q;
        if(q >= p.ntasks) break;
        const uint4 t = p.tasks[q];
        const JobView jv = p.jobs[t.x];
        rows_pair_task<RMAX, W, true>(jv, t.y, t.z, 1, sprof_b, bound, warp, lane);
    }
}

// Pairs that involve a sequence with END units before its last letter, or an
// empty one: the reference's orientation (rows = more 3-unit blocks, ties to
// the pair's second element) and its END handling (rows stop at the first END,
// END columns copy the left neighbour over the full padded width).
template <int R, int WPB>
__global__ void __launch_bounds__(WPB * 32) nw_generic_kernel(NwParams p)
{
    extern __shared__ __align__(16) int8_t smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int8_t *sprof = smem + warp * (kAlpha * 32 * R);
    const uint64_t gw = (uint64_t) blockIdx.x * WPB + warp;
    const uint64_t nw = (uint64_t) gridDim.x * WPB;
    uint32_t *bound = p.bound + gw * p.bound_stride;
    for(uint64_t k = gw; k < p.ngeneric; k += nw) {
        const uint32_t ri = p.gpairs[2 * k], ci = p.gpairs[2 * k + 1];
        const int nrows = (int) p.eff[ri], ncols = (int) p.plen[ci];
        int32_t ra = -ncols * p.g, rb = 0;
        if(nrows > 0 && ncols > 0) {
            dev::run_task<R, dev::Wide, true>(p.prof + p.poff[ri], p.plp[ri], nrows,
                                              p.units + p.uoff[ci], ncols, nullptr, 0,
                                              sprof, bound, p.g, lane, ra, rb);
        } else if(nrows > 0) {
            ra = -nrows * p.g;   // no columns: every row copies column 0
        }
        if(lane == 0) p.out[dev::tri_index(ri, ci)] = ra;
    }
}

// Score profile of every sequence: prof[off + b*Lp + i] = T[unit_i][b] for
// i < eff, 0 beyond. One block per sequence, 16 bytes per thread step.
__global__ void build_profiles_kernel(const uint8_t *__restrict__ units, const uint64_t *__restrict__ uoff,
                                      const uint32_t *__restrict__ eff, const uint64_t *__restrict__ poff,
                                      const uint32_t *__restrict__ plp, const int8_t *__restrict__ ext,
                                      int8_t *__restrict__ prof)
{
    __shared__ int8_t tbl[kAlpha * kAlpha];
    for(int i = threadIdx.x; i < kAlpha * kAlpha; i += blockDim.x) tbl[i] = ext[i];
    __syncthreads();
    const uint32_t s = blockIdx.x;
    const uint8_t *u = units + uoff[s];
    const uint32_t e = eff[s], lp = plp[s];
    int8_t *dst = prof + poff[s];
    const uint32_t chunks = lp / 16;
    for(uint32_t c = threadIdx.x; c < chunks * kAlpha; c += blockDim.x) {
        const uint32_t b = c / chunks, w = c - b * chunks;
        const uint32_t i = w * 16;
        uint32_t out[4] = {0, 0, 0, 0};
        if(i < e) {
            const uint4 v = *reinterpret_cast<const uint4 *>(u + i);
            const uint32_t in[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for(int q = 0; q < 4; ++q) {
#pragma unroll
                for(int k = 0; k < 4; ++k) {
                    const uint32_t x = (in[q] >> (8 * k)) & 0xffu;
                    const int8_t sc = (i + 4 * q + k < e && x < (uint32_t) kAlpha) ? tbl[x * kAlpha + b] : 0;
                    out[q] |= ((uint32_t) (uint8_t) sc) << (8 * k);
                }
            }
        }
        *reinterpret_cast<uint4 *>(dst + (size_t) b * lp + i) = make_uint4(out[0], out[1], out[2], out[3]);
    }
}

// ---------------------------------------------------------------- host side

static constexpr int kPlainR = 16;
static constexpr int kWPB = 4;

template <int R>
static size_t smem_bytes() { return (size_t) kWPB * kAlpha * 32 * R; }

struct Launch {
    int blocks_per_sm = 0;
};

template <class KernelT>
static int occupancy(KernelT kernel, size_t smem, int *blocks)
{
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    if(e != cudaSuccess) return -1;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, kernel, kWPB * 32, smem);
    if(e != cudaSuccess || *blocks < 1) return -1;
    return 0;
}

// 16-bit lanes are exact when every scored cell of a task fits them. In the
// lane state T(i,j) = H(i,j) + g(i+j) every path scores the sum of s + 2g over
// its matched cells, so with smin + 2g >= 0 the state and its diagonal
// candidate lie in [0, min(i,j)*(smax + 2g)], with min(i,j) <= min(rows, cols).
// Cells outside the sequences (padding rows, the shorter sequence's tail) may
// wrap within their half but never feed a scored cell. Clean sequences hold
// letter units only, so smin and smax are taken over the letter block.
static inline bool narrow_ok(int64_t rows_p, int64_t cols, const ExtTable &t)
{
    const int64_t g2 = 2 * (int64_t) t.penalty;
    if((int64_t) t.letter_neg > g2) return false;
    const int64_t step = std::max<int64_t>((int64_t) t.letter_pos + g2, 0);
    if(step > 0xff) return false;   // s + 2g is staged as a byte in packed rows
    return step * std::min(rows_p, cols) <= 0xffff;
}

// Batched-kernel tile shapes (pick_tiles: rows per lane R and warps per CTA
// W) and column groups per single-strip task (pick_chunk), autotuned; the
// context may override either (msa_nw_set_tiles, msa_nw_set_variant).
#include "autotune.inc"

Tiles pick_tiles_for(const SeqStore *st) { return pick_tiles(st, (uint32_t) st->clean_sorted.size()); }

cudaError_t launch_profiles(const SeqStore *st, const int8_t *d_ext, int8_t *d_prof, cudaStream_t s)
{
    if(st->n == 0) return cudaSuccess;
    build_profiles_kernel<<<st->n, 256, 0, s>>>(st->d_units, st->d_off, st->d_eff, st->d_prof_off, st->d_prof_lp,
                                                d_ext, d_prof);
    return cudaGetLastError();
}

void plan_rows_pairs(const SeqStore *st, const ExtTable &tbl, Tiles tiles, std::vector<uint8_t> &narrow,
                     std::vector<uint32_t> &groups)
{
    const uint32_t nclean = (uint32_t) st->clean_sorted.size();
    const uint32_t K = (nclean + 1) / 2;
    const int SH = 32 * tiles.R;
    narrow.assign(K, 0);
    groups.assign(K, 0);
    for(uint32_t k = 0; k < K; ++k) {
        const int64_t ncol = (int64_t) nclean - (2 * (int64_t) k + 1);
        if(ncol <= 0) continue;
        const int64_t rows_p = (int64_t) round_up(st->eff[st->clean_sorted[2 * k]], SH);
        const int64_t cols = st->eff[st->clean_sorted[2 * k + 1]];
        narrow[k] = narrow_ok(rows_p, cols, tbl) ? 1 : 0;
        groups[k] = (uint32_t) ((ncol + tiles.W - 1) / tiles.W);
    }
}

size_t job_view_bytes() { return sizeof(JobView); }

void fill_job_view(void *dst, const SeqStore *st, const int8_t *d_prof, const uint8_t *d_narrow, int32_t *d_out,
                   int32_t g)
{
    JobView v{};
    v.units = st->d_units;
    v.uoff = st->d_off;
    v.eff = st->d_eff;
    v.prof = d_prof;
    v.poff = st->d_prof_off;
    v.plp = st->d_prof_lp;
    v.sorted = st->d_clean_sorted;
    v.row_narrow = d_narrow;
    v.out = d_out;
    v.nclean = (uint32_t) st->clean_sorted.size();
    v.g = g;
    std::memcpy(dst, &v, sizeof(v));
}

cudaError_t load_profiles_kernel()
{
    cudaFuncAttributes a{};
    return cudaFuncGetAttributes(&a, build_profiles_kernel);
}

int serve_grid(msa_ctx *ctx, uint64_t *grid)
{
    auto kern = nw_serve_kernel<32, 8>;
    const size_t smem = (size_t) kAlpha * 32 * 32 * 4;
    MSA_CUDA_TRY(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    int bps = 0;
    MSA_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, 8 * 32, smem));
    if(bps < 1) return set_error(ctx, MSA_ERR_CUDA, "serving kernel cannot be resident");
    *grid = (uint64_t) ctx->num_sms * bps;
    return MSA_OK;
}

cudaError_t launch_serve(const ServeLaunch &l, uint64_t grid, cudaStream_t s)
{
    ServeParams p{};
    p.jobs = (const JobView *) l.jobs;
    p.tasks = (const uint4 *) l.tasks;
    p.ntasks = l.ntasks;
    p.bound = l.bound;
    p.bound_stride = l.bound_stride;
    p.counter = l.counter;
    const size_t smem = (size_t) kAlpha * 32 * 32 * 4;
    nw_serve_kernel<32, 8><<<(unsigned) std::min<uint64_t>(grid, std::max<uint64_t>(l.ntasks, 1)), 8 * 32, smem, s>>>(p);
    return cudaGetLastError();
}


// ---------------------------------------------------------------- plans and graphs
//
// A plan is everything a call needs besides the store: the host-side task
// tables, and device buffers it owns (score profiles, the table, boundary
// rows, task tables, the work counter). Plans are cached per context, keyed by
// store, table, mode, tile shape and output pointer; for the persistent mode
// the launch sequence is captured once into a CUDA graph and replayed.

struct PlainLaunch { uint64_t k_lo, k_hi, blocks; };

struct NwPlan {
    uint64_t store_serial = 0;
    int mode = 0;
    int32_t *d_out = nullptr;
    Tiles tiles{0, 0};
    ExtTable tbl{};
    DevBuf mem;
    const int8_t *d_ext = nullptr;
    NwParams p{};
    BatchParams bp{};
    uint32_t n = 0;
    uint64_t ngeneric = 0, gen_blocks = 0;
    std::vector<PlainLaunch> plain;
    uint64_t batch_grid = 0;
    uint32_t launches = 0, narrow_tasks = 0;
    uint64_t cells = 0, pairs = 0;
    uint32_t part = 0, nparts = 1;
    int variant = 0;            // msa_nw_set_variant flags the plan was built with
    uint32_t chunk = 0;         // and its groups-per-task override
    cudaGraphExec_t exec = nullptr;
    cudaStream_t captured_on = nullptr;
    ~NwPlan()
    {
        if(exec) cudaGraphExecDestroy(exec);
        mem.release();
    }
};

struct GraphCache {
    std::vector<NwPlan *> plans;   // most recent last
};

static constexpr size_t kMaxPlans = 2;

void release_graphs(msa_ctx *ctx)
{
    if(!ctx->graphs) return;
    for(NwPlan *pl : ctx->graphs->plans) delete pl;
    delete ctx->graphs;
    ctx->graphs = nullptr;
}

void drop_plans_for_store(msa_ctx *ctx, uint64_t serial)
{
    if(!ctx->graphs) return;
    auto &v = ctx->graphs->plans;
    for(size_t i = 0; i < v.size();) {
        if(v[i]->store_serial == serial) { delete v[i]; v.erase(v.begin() + i); }
        else ++i;
    }
}

template <int R, int W, bool kPack = true>
static int batched_grid(msa_ctx *ctx, uint64_t ntasks, uint64_t *grid)
{
    auto kern = nw_batched_kernel<R, W, kPack>;
    const size_t smem = (size_t) kAlpha * 32 * R * 4;
    MSA_CUDA_TRY(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    int bps = 0;
    MSA_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, W * 32, smem));
    if(bps < 1) return set_error(ctx, MSA_ERR_CUDA, "batched NW kernel cannot be resident");
    *grid = std::min<uint64_t>((uint64_t) ctx->num_sms * bps, std::max<uint64_t>(ntasks, 1));
    return MSA_OK;
}

template <int R, int W, bool kPack = true>
static void launch_batched(const NwPlan &pl, cudaStream_t s)
{
    const size_t smem = (size_t) kAlpha * 32 * R * 4;
    nw_batched_kernel<R, W, kPack><<<(unsigned) pl.batch_grid, W * 32, smem, s>>>(pl.bp);
}

static int build_plan(msa_ctx *ctx, SeqStore *st, const ExtTable &tbl, int mode, int32_t *d_out, Tiles tiles,
                      uint32_t part, uint32_t nparts, NwPlan *pl)
{
    const uint32_t n = st->n;
    pl->store_serial = st->serial;
    pl->mode = mode;
    pl->d_out = d_out;
    pl->tiles = tiles;
    pl->tbl = tbl;
    pl->n = n;
    pl->part = part;
    pl->nparts = nparts;
    pl->variant = ctx->nw_variant;
    pl->chunk = ctx->nw_chunk;

    const uint32_t nclean = (uint32_t) st->clean_sorted.size();
    const uint64_t nclean_pairs = (uint64_t) nclean * (nclean > 0 ? nclean - 1 : 0) / 2;

    // Pairs with at least one dirty sequence, in the reference's orientation,
    // and this part's runs of rows pairs and generic pairs.
    std::vector<uint32_t> gpairs_all;
    list_generic_pairs(st->dirty, st->len, gpairs_all);
    const JobSplit split = split_job(st->eff, st->plen, st->clean_sorted, gpairs_all, nparts);
    const uint32_t k_lo = split.k[part], k_hi = split.k[part + 1];
    const uint64_t g_lo = split.g[part], g_hi = split.g[part + 1];
    const std::vector<uint32_t> gpairs(gpairs_all.begin() + 2 * g_lo, gpairs_all.begin() + 2 * g_hi);
    pl->ngeneric = gpairs.size() / 2;

    // Pairs and cells (given lengths) of this part.
    {
        using u128 = unsigned __int128;
        const auto &cs = st->clean_sorted;
        std::vector<u128> suffix(nclean + 1, 0);
        for(uint32_t b = nclean; b-- > 0;) suffix[b] = suffix[b + 1] + st->len[cs[b]];
        u128 cells = 0;
        uint64_t pairs = 0;
        for(uint32_t a = 2 * k_lo; a < std::min<uint32_t>(2 * k_hi, nclean); ++a) {
            cells += (u128) st->len[cs[a]] * suffix[a + 1];
            pairs += nclean - 1 - a;
        }
        for(uint64_t q = 0; q < pl->ngeneric; ++q) cells += (u128) st->len[gpairs[2 * q]] * st->len[gpairs[2 * q + 1]];
        pl->cells = (uint64_t) cells;
        pl->pairs = pairs + pl->ngeneric;
    }

    uint32_t max_cols = 1;
    for(uint32_t i = 0; i < n; ++i) max_cols = std::max(max_cols, st->plen[i]);
    const uint64_t stride = round_up((uint64_t) max_cols + 160, 32);

    // Occupancy of the per-warp kernels.
    const size_t smem = smem_bytes<kPlainR>();
    int bps = 0, bps3 = 0;
    if(occupancy(nw_plain_kernel<kPlainR, kWPB>, smem, &bps) || occupancy(nw_generic_kernel<kPlainR, kWPB>, smem, &bps3))
        return set_error(ctx, MSA_ERR_CUDA, "occupancy query failed (no sm_100a image?)");
    bps = std::min(bps, bps3);
    const uint64_t resident_blocks = (uint64_t) ctx->num_sms * (uint64_t) bps;
    uint64_t warps_needed = resident_blocks * kWPB;

    // Persistent task tables: rows pairs (sorted 2k, 2k+1) x column groups of W.
    std::vector<uint64_t> row_task;
    std::vector<uint8_t> row_narrow;
    uint64_t ntasks = 0;
    uint32_t K = 0;
    uint64_t task_base = 0;
    uint32_t gchunk = 1;
    if(mode == MSA_NW_PERSISTENT && nclean_pairs > 0) {
        const int SH = 32 * tiles.R;
        K = (nclean + 1) / 2;
        row_narrow.assign(K, 0);
        std::vector<uint64_t> groups_k(K, 0);
        for(uint32_t k = 0; k < K; ++k) {
            const int64_t ncol = (int64_t) nclean - (2 * (int64_t) k + 1);
            if(ncol <= 0) continue;
            const int64_t rows_p = (int64_t) round_up(st->eff[st->clean_sorted[2 * k]], SH);
            const int64_t cols = st->eff[st->clean_sorted[2 * k + 1]];
            const bool nar = narrow_ok(rows_p, cols, tbl) && !(ctx->nw_variant & MSA_NW_VARIANT_INT32);
            row_narrow[k] = nar ? kRowNarrow : 0;
            groups_k[k] = (uint64_t) (ncol + tiles.W - 1) / tiles.W;
            if(nar && k >= k_lo && k < k_hi) pl->narrow_tasks += (uint32_t) groups_k[k];
        }
        // Short rows pairs two by two in one warp (quad_task): both on 16-bit
        // lanes with the state bound holding for 512 rows, the first's
        // longer sequence within 16 x 32 rows, the second with two sequences
        // and columns, and both in this part. The second's tasks are the
        // first's.
        if(tiles.R == 32 && narrow_ok(512, 512, tbl)) {
            for(uint32_t k = k_lo; k + 1 < k_hi; ++k) {
                if(!(row_narrow[k] && row_narrow[k + 1])) continue;
                if(st->eff[st->clean_sorted[2 * k]] > 16 * 32) continue;
                if(2 * (uint64_t) k + 3 >= nclean) break;
                row_narrow[k] |= kRowQuad;
                groups_k[k + 1] = 0;
                ++k;
            }
        }
        // Tasks of a single-strip rows pair take up to gchunk column groups
        // (one staging of the strip for all of them) while this part keeps at
        // least 16 tasks per resident CTA for the work-stealing tail.
        auto tables = [&](uint32_t chunk) {
            row_task.assign(K + 1, 0);
            uint64_t nt = 0;
            for(uint32_t k = 0; k < K; ++k) {
                row_task[k] = nt;
                const uint32_t c = groups_per_task(st->eff[st->clean_sorted[2 * k]], tiles.R, chunk);
                nt += (groups_k[k] + c - 1) / c;
            }
            row_task[K] = nt;
            return row_task[k_hi] - row_task[k_lo];
        };
        int rc;
        const uint64_t all_groups = tables(1);
        if(ctx->nw_variant & MSA_NW_VARIANT_NO_PACKED) rc = batched_grid<32, 8, false>(ctx, all_groups, &pl->batch_grid);
        else if(tiles.R == 16 && tiles.W == 4) rc = batched_grid<16, 4>(ctx, all_groups, &pl->batch_grid);
        else if(tiles.R == 16 && tiles.W == 8) rc = batched_grid<16, 8>(ctx, all_groups, &pl->batch_grid);
        else if(tiles.R == 32 && tiles.W == 4) rc = batched_grid<32, 4>(ctx, all_groups, &pl->batch_grid);
        else rc = batched_grid<32, 8>(ctx, all_groups, &pl->batch_grid);
        if(rc) return rc;
        const uint32_t want = ctx->nw_chunk ? ctx->nw_chunk : pick_chunk(st, nclean);
        for(gchunk = want; gchunk > 1 && tables(gchunk) < 16 * pl->batch_grid; gchunk /= 2) {}
        ntasks = tables(gchunk);
        // This part's tasks: those of rows pairs [k_lo, k_hi).
        task_base = row_task[k_lo];
        warps_needed = std::max<uint64_t>(warps_needed, pl->batch_grid * tiles.W);
    }

    // One device allocation owned by the plan.
    size_t off = 0;
    auto take = [&off](size_t b) { size_t o = off; off = round_up(off + b, 256); return o; };
    const size_t o_prof = take(st->prof_bytes + 64), o_ext = take(kAlpha * kAlpha),
                 o_bound = take(warps_needed * stride * sizeof(uint32_t)), o_rt = take((K + 1) * sizeof(uint64_t)),
                 o_rn = take(K + 16), o_gp = take(gpairs.size() * sizeof(uint32_t) + 16), o_cnt = take(64);
    MSA_CUDA_TRY(ctx, pl->mem.ensure(off));
    char *base = (char *) pl->mem.ptr;
    cudaStream_t s = ctx->stream;
    MSA_CUDA_TRY(ctx, cudaMemcpyAsync(base + o_ext, tbl.score, kAlpha * kAlpha, cudaMemcpyHostToDevice, s));
    if(K) {
        MSA_CUDA_TRY(ctx, cudaMemcpyAsync(base + o_rt, row_task.data(), (K + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
        MSA_CUDA_TRY(ctx, cudaMemcpyAsync(base + o_rn, row_narrow.data(), K, cudaMemcpyHostToDevice, s));
    }
    if(!gpairs.empty())
        MSA_CUDA_TRY(ctx, cudaMemcpyAsync(base + o_gp, gpairs.data(), gpairs.size() * sizeof(uint32_t),
                                          cudaMemcpyHostToDevice, s));
    MSA_CUDA_TRY(ctx, cudaStreamSynchronize(s));   // host vectors go out of scope

    pl->d_ext = (const int8_t *) (base + o_ext);
    NwParams &p = pl->p;
    p.units = st->d_units;
    p.uoff = st->d_off;
    p.eff = st->d_eff;
    p.plen = st->d_plen;
    p.prof = (const int8_t *) (base + o_prof);
    p.poff = st->d_prof_off;
    p.plp = st->d_prof_lp;
    p.sorted = st->d_clean_sorted;
    p.nclean = nclean;
    p.out = d_out;
    p.g = tbl.penalty;
    p.bound_stride = stride;
    p.bound = (uint32_t *) (base + o_bound);
    p.gpairs = (const uint32_t *) (base + o_gp);
    p.ngeneric = pl->ngeneric;
    pl->gen_blocks = std::min<uint64_t>(resident_blocks, (pl->ngeneric + kWPB - 1) / kWPB);

    BatchParams &bp = pl->bp;
    bp.job.units = st->d_units;
    bp.job.uoff = st->d_off;
    bp.job.eff = st->d_eff;
    bp.job.prof = p.prof;
    bp.job.poff = st->d_prof_off;
    bp.job.plp = st->d_prof_lp;
    bp.job.sorted = st->d_clean_sorted;
    bp.job.nclean = nclean;
    bp.job.row_narrow = (const uint8_t *) (base + o_rn);
    bp.job.out = d_out;
    bp.job.g = tbl.penalty;
    bp.npairs_rows = K;
    bp.row_task = (const uint64_t *) (base + o_rt);
    bp.ntasks = ntasks;
    bp.task_base = task_base;
    bp.gchunk = gchunk;
    bp.bound = p.bound;
    bp.bound_stride = stride;
    bp.counter = (unsigned long long *) (base + o_cnt);

    pl->launches = 1 + (pl->ngeneric ? 1 : 0);
    if(mode == MSA_NW_PLAIN && nclean_pairs > 0) {
        // Buckets: runs of sorted rows with the same strip count.
        constexpr int SH = 32 * kPlainR;
        // This part's rows: sorted [2 k_lo, 2 k_hi).
        const uint32_t a_end = std::min<uint32_t>(2 * k_hi, nclean);
        uint32_t a = std::min<uint32_t>(2 * k_lo, nclean);
        while(a < a_end && a + 1 < nclean) {
            const uint32_t strips = (st->eff[st->clean_sorted[a]] + SH - 1) / SH;
            uint32_t a2 = a + 1;
            while(a2 < a_end && a2 + 1 < nclean && (st->eff[st->clean_sorted[a2]] + SH - 1) / SH == strips) ++a2;
            const uint64_t k_lo = (uint64_t) a * (2 * (uint64_t) nclean - a - 1) / 2;
            const uint64_t k_hi = (uint64_t) a2 * (2 * (uint64_t) nclean - a2 - 1) / 2;
            pl->plain.push_back({k_lo, k_hi, std::min<uint64_t>(resident_blocks, (k_hi - k_lo + kWPB - 1) / kWPB)});
            a = a2;
        }
        pl->launches += (uint32_t) pl->plain.size();
    } else if(ntasks > 0) {
        pl->launches += 1;
    }
    return MSA_OK;
}

// Enqueues one scoring pass. Events are recorded with cudaEventRecordExternal
// while capturing so they stay real timing records inside the graph.
static cudaError_t enqueue(msa_ctx *ctx, const NwPlan &pl, const SeqStore *st, cudaStream_t s, bool capturing)
{
    const unsigned flags = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    cudaError_t e = cudaEventRecordWithFlags(ctx->ev[0], s, flags);
    if(e) return e;
    build_profiles_kernel<<<pl.n, 256, 0, s>>>(st->d_units, st->d_off, st->d_eff, st->d_prof_off, st->d_prof_lp,
                                               pl.d_ext, const_cast<int8_t *>(pl.p.prof));
    if((e = cudaGetLastError())) return e;
    if((e = cudaEventRecordWithFlags(ctx->ev[1], s, flags))) return e;
    const size_t smem = smem_bytes<kPlainR>();
    if(pl.ngeneric) {
        nw_generic_kernel<kPlainR, kWPB><<<(unsigned) pl.gen_blocks, kWPB * 32, smem, s>>>(pl.p);
        if((e = cudaGetLastError())) return e;
    }
    if(pl.mode == MSA_NW_PLAIN) {
        for(const PlainLaunch &L : pl.plain) {
            nw_plain_kernel<kPlainR, kWPB><<<(unsigned) L.blocks, kWPB * 32, smem, s>>>(pl.p, L.k_lo, L.k_hi);
            if((e = cudaGetLastError())) return e;
        }
    } else if(pl.bp.ntasks) {
        if((e = cudaMemsetAsync(pl.bp.counter, 0, 64, s))) return e;
        const Tiles t = pl.tiles;
        if(pl.variant & MSA_NW_VARIANT_NO_PACKED) launch_batched<32, 8, false>(pl, s);
        else if(t.R == 16 && t.W == 4) launch_batched<16, 4>(pl, s);
        else if(t.R == 16 && t.W == 8) launch_batched<16, 8>(pl, s);
        else if(t.R == 32 && t.W == 4) launch_batched<32, 4>(pl, s);
        else launch_batched<32, 8>(pl, s);
        if((e = cudaGetLastError())) return e;
    }
    return cudaEventRecordWithFlags(ctx->ev[2], s, flags);
}

static bool same_table(const ExtTable &a, const ExtTable &b)
{
    return std::memcmp(a.score, b.score, sizeof(a.score)) == 0 && std::memcmp(a.valid, b.valid, sizeof(a.valid)) == 0 &&
           a.penalty == b.penalty;
}

int nw_run(msa_ctx *ctx, SeqStore *st, const ExtTable &tbl, int mode, int32_t *d_out, uint32_t part,
           uint32_t nparts)
{
    cudaStream_t s = ctx->stream;
    const uint32_t n = st->n;
    msa_nw_stats stats{};
    stats.pairs = (uint64_t) n * (n > 0 ? n - 1 : 0) / 2;
    if(n < 2) { ctx->last = stats; return MSA_OK; }

    const uint32_t nclean = (uint32_t) st->clean_sorted.size();
    const Tiles tiles = mode != MSA_NW_PERSISTENT ? Tiles{0, 0}
                      : (ctx->nw_variant & MSA_NW_VARIANT_NO_PACKED) ? Tiles{32, 8}
                      : ctx->tile_r ? Tiles{ctx->tile_r, ctx->tile_w} : pick_tiles(st, nclean);

    if(!ctx->graphs) ctx->graphs = new GraphCache;
    auto &plans = ctx->graphs->plans;
    NwPlan *pl = nullptr;
    for(size_t i = 0; i < plans.size(); ++i) {
        NwPlan *c = plans[i];
        if(c->store_serial == st->serial && c->mode == mode && c->d_out == d_out && c->tiles.R == tiles.R &&
           c->tiles.W == tiles.W && c->part == part && c->nparts == nparts && same_table(c->tbl, tbl) &&
           c->variant == ctx->nw_variant && c->chunk == ctx->nw_chunk) {
            pl = c;
            plans.erase(plans.begin() + i);
            plans.push_back(pl);
            break;
        }
    }
    if(!pl) {
        while(plans.size() >= kMaxPlans) { delete plans.front(); plans.erase(plans.begin()); }
        pl = new NwPlan;
        const int rc = build_plan(ctx, st, tbl, mode, d_out, tiles, part, nparts, pl);
        if(rc) { delete pl; return rc; }
        plans.push_back(pl);
    }

    // The persistent mode replays a captured graph; the legacy default stream
    // cannot be captured, so there the same sequence is launched directly.
    bool use_graph = mode == MSA_NW_PERSISTENT && s != nullptr;
    if(use_graph && (!pl->exec || pl->captured_on != s)) {
        if(pl->exec) { cudaGraphExecDestroy(pl->exec); pl->exec = nullptr; }
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if(!e) {
            const cudaError_t e2 = enqueue(ctx, *pl, st, s, true);
            e = cudaStreamEndCapture(s, &g);
            if(!e) e = e2;
        }
        if(!e) e = cudaGraphInstantiate(&pl->exec, g, 0);
        if(g) cudaGraphDestroy(g);
        if(e) {
            cudaGetLastError();
            pl->exec = nullptr;
            use_graph = false;   // launch the same kernels directly
        } else {
            pl->captured_on = s;
        }
    }
    if(use_graph) {
        MSA_CUDA_TRY(ctx, cudaGraphLaunch(pl->exec, s));
    } else {
        MSA_CUDA_TRY(ctx, enqueue(ctx, *pl, st, s, false));
    }
    ctx->launches += pl->launches;

    MSA_CUDA_TRY(ctx, cudaEventSynchronize(ctx->ev[2]));
    float ms_k = 0, ms_t = 0;
    cudaEventElapsedTime(&ms_k, ctx->ev[1], ctx->ev[2]);
    cudaEventElapsedTime(&ms_t, ctx->ev[0], ctx->ev[2]);
    stats.kernel_ms = ms_k;
    stats.total_ms = ms_t;
    stats.cells = pl->cells;
    stats.launches = pl->launches;
    stats.narrow_tasks = pl->narrow_tasks;
    stats.graph = use_graph ? 1 : 0;
    ctx->last = stats;
    return MSA_OK;
}

}  // namespace msa
