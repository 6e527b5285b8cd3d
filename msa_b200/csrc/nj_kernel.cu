// Neighbor-joining on the device, bit-exact with the reference's
// njoining::sequential<transform::symmetric>
// (src/phylogeny/njoining/impl/sequential.cpp:80-346).
//
// The reference shrinks a packed symmetric matrix after every join (swap the
// removed OTU with logical 0, then drop logical 0: src/phylogeny/matrix.cu:359-384,
// sequential.cpp:210-224). Here the matrix never moves: D is a full n x n
// float matrix indexed by physical slot, and a logical -> physical permutation
// reproduces the reference's index order, which is what its first-maximum
// tie-break scans. Every float and double operation is written out with an
// explicit rounding intrinsic in the reference's order, so no FMA contraction
// or reassociation can change a bit.
//
// One cooperative launch runs all joins. While many OTUs remain, every block
// scans a slice of the logical lower triangle (Q = (c-2)*D - S_i - S_j) for its
// (max Q, first index) candidate, a grid barrier publishes the slices, every
// block reduces them identically, block 0 applies the join, and a second
// barrier releases the next scan. Once few OTUs remain, block 0 finishes alone
// with block-level barriers only. Every grid-barrier wait is bounded: on
// timeout the kernel raises an error flag and all blocks return.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include <cooperative_groups.h>

#include "msa_internal.hpp"

namespace msa {
namespace njdev {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kThreads = 1024;
constexpr unsigned long long kSpinLimit = 1ull << 24;   // x 64 ns sleeps ~ 1 s

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

// Larger Q wins; on equal Q the smaller row-major index (earlier in the
// reference's scan) wins.
__device__ __forceinline__ unsigned long long pack(uint32_t key, uint32_t lin)
{
    return key ? (((unsigned long long) key << 32) | (0xffffffffu - lin)) : 0ull;
}

__device__ __forceinline__ unsigned long long umax64(unsigned long long a, unsigned long long b) { return a > b ? a : b; }

__device__ __forceinline__ unsigned long long warp_max(unsigned long long v)
{
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) v = umax64(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

struct State {
    float *D;                // n x n, physical slots
    float *S;                // row sums by physical slot
    uint32_t *perm[2];       // logical -> physical, double buffered
    uint32_t *map;           // OTU id by physical slot
    unsigned long long *partial;
    uint32_t *rec_x, *rec_y; // OTU ids joined at each step
    float *rec_dx, *rec_dy;
    unsigned *bar;
    int *err;
    unsigned long long *cycles;   // 6 phase counters written by block 0
    uint32_t n;
    uint32_t single_c;       // block 0 continues alone once c <= single_c
};

__device__ __forceinline__ bool grid_sync(unsigned *bar, unsigned nblocks, unsigned &epoch, int *err)
{
    __syncthreads();
    if(threadIdx.x == 0) {
        ++epoch;
        __threadfence();
        atomicAdd(bar, 1u);
        const unsigned target = epoch * nblocks;
        unsigned long long spins = 0;
        for(;;) {
            unsigned v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
            if(v >= target) break;
            if(*(volatile int *) err) break;
            if(++spins > kSpinLimit) { atomicExch(err, 1); break; }
            __nanosleep(20);
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int *) err == 0;
}

// Row-major lower-triangle index -> (i, j), i > j.
__device__ __forceinline__ void tri_decode(uint64_t L, uint32_t &i, uint32_t &j)
{
    uint64_t r = (uint64_t) ((1.0 + sqrt(1.0 + 8.0 * (double) L)) * 0.5);
    while(r * (r - 1) / 2 > L) --r;
    while((r + 1) * r / 2 <= L) ++r;
    i = (uint32_t) r;
    j = (uint32_t) (L - r * (r - 1) / 2);
}

// Best (Q, row-major index) of rows gw, gw + nwt, ... of the logical lower
// triangle. kCG: other blocks write D, so loads bypass L1.
template <bool kCG>
__device__ __forceinline__ void scan_rows(const float *__restrict__ D, uint32_t n, const uint32_t *pl, const float *Sl,
                                          uint32_t c, float cm2, uint32_t gw, uint32_t nwt, int lane, float &bq,
                                          uint32_t &bl)
{
    for(uint32_t i = 1 + gw; i < c; i += nwt) {
        const float *row = D + (size_t) pl[i] * n;
        const float si = Sl[i];
        const uint32_t base = i * (i - 1) / 2;
        for(uint32_t j = lane; j < i; j += 32) {
            const float d = kCG ? __ldcg(row + pl[j]) : row[pl[j]];
            const float q = __fsub_rn(__fsub_rn(__fmul_rn(cm2, d), si), Sl[j]);
            if(q > bq) { bq = q; bl = base + j; }
        }
    }
}

__global__ void __launch_bounds__(kThreads) nj_kernel(State st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t n = st.n;
    // Shared layout (16-byte aligned regions): logical -> physical slots, S in
    // logical order (reused for the float row-sum updates once a join has read
    // it), and block 0's double-precision updates.
    const size_t off_s = ((size_t) n * 4 + 15) & ~(size_t) 15;
    const size_t off_u = (off_s + (size_t) n * 4 + 15) & ~(size_t) 15;
    uint32_t *pl = reinterpret_cast<uint32_t *>(smem_raw);
    float *Sl = reinterpret_cast<float *>(smem_raw + off_s);
    double *upd = reinterpret_cast<double *>(smem_raw + off_u);
    __shared__ unsigned long long wbest[kThreads / 32];
    __shared__ unsigned long long chosen;
    __shared__ uint8_t exact_all;

    const unsigned nblocks = gridDim.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned epoch = 0;
    // Block 0, thread 0: cycles spent per phase (grid: scan, wait, join, wait;
    // single: scan, join) for msa_nj_last_stats.
    unsigned long long cyc[6] = {0, 0, 0, 0, 0, 0};
    unsigned long long t_last = clock64();
    auto mark = [&](int k) {
        const unsigned long long t = clock64();
        cyc[k] += t - t_last;
        t_last = t;
    };
    uint32_t c = n;
    int buf = 0;
    uint32_t next_parent = n;
    uint32_t step = 0;

    while(c > 1) {
        const bool single = c <= st.single_c;
        if(single && blockIdx.x != 0) return;
        const uint32_t *perm = buf ? st.perm[1] : st.perm[0];

        for(uint32_t k = tid; k < c; k += kThreads) {
            const uint32_t p = __ldcg(perm + k);
            pl[k] = p;
            Sl[k] = __ldcg(st.S + p);
        }
        __syncthreads();

        // ---- scan: warps take rows i = 1..c-1 round-robin; lanes stride over
        // j < i. Each thread visits its pairs in increasing row-major index, so
        // a strict `>` keeps its first maximum, as the reference's scan does.
        const float cm2 = (float) (c - 2);
        const uint32_t nwt = (single ? 1u : nblocks) * (kThreads / 32);
        const uint32_t gw = (single ? 0u : blockIdx.x) * (kThreads / 32) + warp;
        float bq = -INFINITY;
        uint32_t bl = 0;
        if(single) scan_rows<false>(st.D, n, pl, Sl, c, cm2, gw, nwt, lane, bq, bl);
        else scan_rows<true>(st.D, n, pl, Sl, c, cm2, gw, nwt, lane, bq, bl);
        unsigned long long best = pack(order_key(bq), bl);
        if(blockIdx.x == 0 && tid == 0) mark(single ? 4 : 0);
        best = warp_max(best);
        if(lane == 0) wbest[warp] = best;
        __syncthreads();
        if(warp == 0) {
            unsigned long long v = wbest[lane];
            v = warp_max(v);
            if(lane == 0) {
                if(single) chosen = v;
                else __stcg(st.partial + blockIdx.x, v);
            }
        }
        if(!single) {
            if(!grid_sync(st.bar, nblocks, epoch, st.err)) return;
            if(blockIdx.x == 0 && tid == 0) mark(1);
            if(warp == 0) {
                unsigned long long v = 0;
                for(unsigned b = lane; b < nblocks; b += 32) v = umax64(v, __ldcg(st.partial + b));
                v = warp_max(v);
                if(lane == 0) chosen = v;
            }
        }
        __syncthreads();
        const unsigned long long win = chosen;
        if(win == 0ull) {   // no selectable Q (all NaN): the reference would index an undefined pair
            if(tid == 0) atomicExch(st.err, 2);
            return;
        }

        // ---- join (block 0 only; the others wait at the next barrier).
        if(blockIdx.x == 0) {
            const uint32_t lin = 0xffffffffu - (uint32_t) (win & 0xffffffffull);
            uint32_t x, y;
            tri_decode(lin, x, y);
            const uint32_t px = pl[x], py = pl[y];
            const float dxy = __ldcg(st.D + (size_t) px * n + py);

            // raise_candidate (sequential.cpp:142-152).
            if(tid == 0) {
                const float pairsum = __fsub_rn(Sl[x], Sl[y]);
                const float den = (float) (2u * (c - 2));
                const float q = __fdiv_rn(pairsum, den);
                float dx = __double2float_rn(__dadd_rn(__dmul_rn(0.5, (double) dxy), (double) q));
                float dy = __fsub_rn(dxy, dx);
                // The last join divides by 2(c-2) = 0; for 0/0 the reference's x86
                // SSE arithmetic yields the default NaN 0xFFC00000 and propagates it
                // into dx and dy, where the GPU would give its canonical 0x7FFFFFFF.
                if(dx != dx) dx = __uint_as_float(0xFFC00000u);
                if(dy != dy) dy = __uint_as_float(0xFFC00000u);
                st.rec_x[step] = __ldcg(st.map + px);
                st.rec_y[step] = __ldcg(st.map + py);
                st.rec_dx[step] = dx;
                st.rec_dy[step] = dy;
                exact_all = 1;
            }
            __syncthreads();

            // join_pair (sequential.cpp:247-267): per-row updates.
            bool exact = true;
            for(uint32_t i = tid; i < c; i += kThreads) {
                const uint32_t p = pl[i];
                float a, b;
                if(i == x) { a = __ldcg(st.D + (size_t) px * n + px); b = dxy; }
                else if(i == y) { a = dxy; b = __ldcg(st.D + (size_t) py * n + py); }
                else { a = __ldcg(st.D + (size_t) p * n + px); b = __ldcg(st.D + (size_t) p * n + py); }
                const float prev = __fadd_rn(a, b);
                const double u = __dmul_rn((double) __fsub_rn(prev, dxy), 0.5);
                upd[i] = u;
                exact = exact && ((double) __double2float_rn(u) == u);
                const float nd = __double2float_rn(u);
                __stcg(st.D + (size_t) p * n + px, nd);
                __stcg(st.D + (size_t) px * n + p, nd);
                if(i != x) {
                    const float s = __double2float_rn(__dadd_rn((double) Sl[i], __dsub_rn(u, (double) prev)));
                    __stcg(st.S + p, s);
                }
                Sl[i] = nd;   // this thread's own slot: S[i] was read just above
            }
            if(!exact) exact_all = 0;
            __syncthreads();

            // Serial fold of the new row sum (sequential.cpp:259): i ascending.
            // When every update is a float value, the double add rounded to float
            // equals a float add (double has >= 2*24+2 significand bits), so the
            // short-latency float chain is used; otherwise the literal double one.
            if(tid == 0) {
                float ns = 0.0f;
                if(exact_all) {
                    // Prefetched float4 batches keep the loads off the add chain.
                    const float4 *v4 = reinterpret_cast<const float4 *>(Sl);
                    const uint32_t c4 = c / 4;
                    float4 a = c4 > 0 ? v4[0] : make_float4(0, 0, 0, 0);
                    float4 b = c4 > 1 ? v4[1] : make_float4(0, 0, 0, 0);
                    for(uint32_t q = 0; q < c4; ++q) {
                        const float4 cur = a;
                        a = b;
                        if(q + 2 < c4) b = v4[q + 2];
                        ns = __fadd_rn(ns, cur.x);
                        ns = __fadd_rn(ns, cur.y);
                        ns = __fadd_rn(ns, cur.z);
                        ns = __fadd_rn(ns, cur.w);
                    }
                    for(uint32_t i = 4 * c4; i < c; ++i) ns = __fadd_rn(ns, Sl[i]);
                } else {
                    for(uint32_t i = 0; i < c; ++i) ns = __double2float_rn(__dadd_rn((double) ns, upd[i]));
                }
                __stcg(st.S + px, ns);
                __stcg(st.map + px, next_parent);
            } else {
                // update_cache, symmetric (sequential.cpp:210-224): logical 0 and y
                // swap, then logical 0 is dropped.
                uint32_t *np = buf ? st.perm[0] : st.perm[1];
                for(uint32_t k = tid - 1; k + 1 < c; k += kThreads - 1) {
                    const uint32_t v = (y > 0 && k == y - 1) ? pl[0] : pl[k + 1];
                    __stcg(np + k, v);
                }
            }
        }
        ++next_parent;
        ++step;
        buf ^= 1;
        --c;
        if(blockIdx.x == 0 && tid == 0) mark(single ? 5 : 2);
        if(!single) {
            if(!grid_sync(st.bar, nblocks, epoch, st.err)) return;
            if(blockIdx.x == 0 && tid == 0) mark(3);
        } else {
            __threadfence_block();
            __syncthreads();
        }
    }
    if(blockIdx.x == 0 && tid == 0)
        for(int k = 0; k < 6; ++k) st.cycles[k] = cyc[k];
}

// Packed triangle (float or int32) -> full symmetric matrix, diagonal 0.
template <class T>
__global__ void inflate_kernel(const T *__restrict__ tri, float *__restrict__ D, uint32_t n)
{
    const uint64_t total = (uint64_t) n * n;
    for(uint64_t e = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t) gridDim.x * blockDim.x) {
        const uint64_t i = e / n, j = e - i * n;
        float v = 0.0f;
        if(i > j) v = (float) tri[i * (i - 1) / 2 + j];
        else if(j > i) v = (float) tri[j * (j - 1) / 2 + i];
        D[e] = v;
    }
}

// cache_init (sequential.cpp:80-94): S[k] folds D[k][j] over j != k ascending,
// from 0. Thread k reads column k (= row k by symmetry) so a warp's reads coalesce.
__global__ void row_sums_kernel(const float *__restrict__ D, float *__restrict__ S, uint32_t *perm,
                                uint32_t *map, uint32_t n)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if(k >= n) return;
    float s = 0.0f;
    for(uint32_t j = 0; j < n; ++j)
        if(j != k) s = __fadd_rn(s, D[(size_t) j * n + k]);
    S[k] = s;
    perm[k] = k;
    map[k] = k;
}

}  // namespace njdev

int nj_run(msa_ctx *ctx, const void *tri, int kind, uint32_t n, msa_otu *out)
{
    cudaStream_t s = ctx->stream;
    const size_t smem = (size_t) n * 16 + 32;   // pl, Sl (4 B each), upd (8 B), alignment
    if(smem > 200 * 1024) return set_error(ctx, MSA_ERR_TOO_LARGE, "neighbor-joining supports at most 12800 OTUs");
    const uint64_t ntri = (uint64_t) n * (n - 1) / 2;

    // Device layout.
    size_t off = 0;
    auto take = [&off](size_t b) { size_t o = off; off = round_up(off + b, 256); return o; };
    const size_t oD = take((size_t) n * n * 4), oS = take(n * 4), oP0 = take(n * 4), oP1 = take(n * 4),
                 oM = take(n * 4), oPart = take(4096 * 8), oRx = take(n * 4), oRy = take(n * 4),
                 oRdx = take(n * 4), oRdy = take(n * 4), oBar = take(64), oErr = take(64), oCyc = take(64),
                 oTri = take((kind == MSA_TRI_F32_HOST || kind == MSA_TRI_I32_HOST) ? ntri * 4 : 0);
    MSA_CUDA_TRY(ctx, ctx->nj_buf.ensure(off));
    char *base = (char *) ctx->nj_buf.ptr;
    njdev::State st{};
    st.D = (float *) (base + oD);
    st.S = (float *) (base + oS);
    st.perm[0] = (uint32_t *) (base + oP0);
    st.perm[1] = (uint32_t *) (base + oP1);
    st.map = (uint32_t *) (base + oM);
    st.partial = (unsigned long long *) (base + oPart);
    st.rec_x = (uint32_t *) (base + oRx);
    st.rec_y = (uint32_t *) (base + oRy);
    st.rec_dx = (float *) (base + oRdx);
    st.rec_dy = (float *) (base + oRdy);
    st.bar = (unsigned *) (base + oBar);
    st.err = (int *) (base + oErr);
    st.cycles = (unsigned long long *) (base + oCyc);
    st.n = n;

    MSA_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[0], s));
    const void *dtri = tri;
    if(kind == MSA_TRI_F32_HOST || kind == MSA_TRI_I32_HOST) {
        MSA_CUDA_TRY(ctx, cudaMemcpyAsync(base + oTri, tri, ntri * 4, cudaMemcpyHostToDevice, s));
        dtri = base + oTri;
    }
    const unsigned ib = (unsigned) std::min<uint64_t>(((uint64_t) n * n + 255) / 256, 65535);
    if(kind == MSA_TRI_F32_HOST || kind == MSA_TRI_F32_DEVICE)
        njdev::inflate_kernel<float><<<ib, 256, 0, s>>>((const float *) dtri, st.D, n);
    else
        njdev::inflate_kernel<int32_t><<<ib, 256, 0, s>>>((const int32_t *) dtri, st.D, n);
    MSA_CUDA_TRY(ctx, cudaGetLastError());
    njdev::row_sums_kernel<<<(n + 255) / 256, 256, 0, s>>>(st.D, st.S, st.perm[0], st.map, n);
    MSA_CUDA_TRY(ctx, cudaGetLastError());
    MSA_CUDA_TRY(ctx, cudaMemsetAsync(base + oBar, 0, 64, s));
    MSA_CUDA_TRY(ctx, cudaMemsetAsync(base + oErr, 0, 64, s));
    ctx->launches += 2;

    MSA_CUDA_TRY(ctx, cudaFuncSetAttribute(njdev::nj_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    int per_sm = 0;
    MSA_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, njdev::nj_kernel, njdev::kThreads, smem));
    if(per_sm < 1) return set_error(ctx, MSA_ERR_CUDA, "neighbor-joining kernel cannot be resident");
    unsigned grid = (unsigned) ctx->num_sms;   // one block per SM; co-resident by cooperative launch
    // Small problems: one block does everything.
    st.single_c = 1024;
    if(n <= st.single_c) grid = 1;
    void *args[] = {&st};
    MSA_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[1], s));
    MSA_CUDA_TRY(ctx, cudaLaunchCooperativeKernel((const void *) njdev::nj_kernel, dim3(grid), dim3(njdev::kThreads),
                                                  args, smem, s));
    MSA_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[2], s));
    ctx->launches++;
    unsigned long long cyc[6] = {0, 0, 0, 0, 0, 0};

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
        ns.grid_joins = n > st.single_c ? n - st.single_c : 0;
        ns.cycles_scan = cyc[0];
        ns.cycles_wait = cyc[1] + cyc[3];
        ns.cycles_join = cyc[2];
        ns.cycles_scan_single = cyc[4];
        ns.cycles_join_single = cyc[5];
        ctx->nj_last = ns;
    }
    if(err == 1) return set_error(ctx, MSA_ERR_DEVICE_TIMEOUT, "neighbor-joining grid barrier timed out");
    if(err == 2) return set_error(ctx, MSA_ERR_UNDEFINED, "no joinable pair: every Q value is NaN");

    // star tree (src/phylogeny/njoining/star.cuh:61-72).
    const uint32_t nodes = 2 * n - 1;
    for(uint32_t k = 0; k < nodes; ++k) {
        out[k].parent = out[k].child[0] = out[k].child[1] = 0xffffffffu;
        out[k].distance = FLT_MAX;
        out[k].level = 0;
    }
    for(uint32_t k = 0; k + 1 < n; ++k) {
        const uint32_t parent = n + k;
        const uint32_t a = rx[k], b = ry[k];
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
