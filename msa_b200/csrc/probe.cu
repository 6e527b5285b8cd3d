// Integer-op throughput probes for the issue roofline: each probe runs eight
// independent dependency chains of one operation form per thread, enough
// warps to fill every SM, and reports lane-operations per SM per clock
// (clock64 deltas inside the kernel, so the figure does not depend on the
// clock the GPU happens to run at).
#include <algorithm>

#include "msa_internal.hpp"

namespace msa {
namespace probe {

template <int OP>
__device__ __forceinline__ uint32_t op(uint32_t a, uint32_t b, uint32_t c)
{
    if constexpr(OP == 0) return a + b;                                               // IADD
    else if constexpr(OP == 1) return (uint32_t) max((int) a, (int) b);              // IMNMX
    else if constexpr(OP == 2) return (uint32_t) __viaddmax_s32((int) a, (int) c, (int) b);
    else if constexpr(OP == 3) return (uint32_t) __vimax3_s32((int) a, (int) b, (int) c);
    else if constexpr(OP == 4) return __vadd2(a, b);
    else if constexpr(OP == 5) return __viaddmax_s16x2(a, c, b);
    else if constexpr(OP == 6) return __vimax3_s16x2(a, b, c);
    else if constexpr(OP == 7) return __viaddmax_u16x2(a, c, b);
    else if constexpr(OP == 8) return __vimax3_u16x2(a, b, c);
    else if constexpr(OP == 9) return __vmaxu2(a, b);
    else if constexpr(OP == 10) {
        uint32_t r;
        asm("prmt.b32 %0, %1, %2, 0xC480;" : "=r"(r) : "r"(a), "r"(b));
        return r;
    } else if constexpr(OP == 11) {
        // The 32-bit NW cell: max(up - g, max(left - g, diag + s)).
        const int ds = (int) a + (int) c;
        const int t = __viaddmax_s32((int) b, -3, ds);
        return (uint32_t) __viaddmax_s32((int) a, -3, t);
    } else if constexpr(OP == 12) {
        // The 16x2 NW cell on signed halves.
        const uint32_t ds = __vadd2(a, c);
        const uint32_t t = __viaddmax_s16x2(b, 0xfffdfffdu, ds);
        return __viaddmax_s16x2(a, 0xfffdfffdu, t);
    } else if constexpr(OP == 13) {
        // The 16x2 NW cell on biased unsigned halves with a 32-bit score add.
        const uint32_t ds = a + c;
        const uint32_t t = __viaddmax_u16x2(b, 0xfffdfffdu, ds);
        return __viaddmax_u16x2(a, 0xfffdfffdu, t);
    } else if constexpr(OP == 14) {
        // The 16x2 NW cell on the gap-free state T = H + g(i+j):
        // max(T_left, T_up, T_diag + s + 2g).
        return __vimax3_u16x2(a, b, __vadd2(b, c));
    } else {
        return a ^ b;
    }
}

template <int OP>
__global__ void __launch_bounds__(256) probe_kernel(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                                                    int iters, unsigned long long *cycles)
{
    uint32_t x[8], y[8];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for(int k = 0; k < 8; ++k) {
        x[k] = in[(t * 16 + k) & 4095];
        y[k] = in[(t * 16 + 8 + k) & 4095];
    }
    __syncthreads();
    const unsigned long long c0 = clock64();
    for(int it = 0; it < iters; ++it) {
#pragma unroll
        for(int k = 0; k < 8; ++k) x[k] = op<OP>(x[k], x[(k + 1) & 7], y[k]);
    }
    __syncthreads();
    const unsigned long long c1 = clock64();
    uint32_t acc = 0;
#pragma unroll
    for(int k = 0; k < 8; ++k) acc ^= x[k];
    out[t] = acc;
    if(threadIdx.x == 0) atomicMax(cycles, c1 - c0);
}

// Shared-memory load bandwidth: every warp reads 512 contiguous bytes per
// ld.shared.v4 (bank-conflict free, the access shape of the NW profile loads),
// eight loads per iteration at addresses that change every iteration.
// ops_per_clk_sm reports bytes per SM per clock.
__global__ void __launch_bounds__(256) probe_lds_kernel(uint32_t *__restrict__ out, int iters,
                                                        unsigned long long *cycles)
{
    __shared__ __align__(16) uint32_t buf[4096];   // 16 KB
    for(int k = threadIdx.x; k < 4096; k += blockDim.x) buf[k] = k * 2654435761u;
    __syncthreads();
    const uint32_t base = (uint32_t) __cvta_generic_to_shared(buf) + (threadIdx.x & 31) * 16;
    uint32_t acc = 0;
    const unsigned long long c0 = clock64();
    for(int it = 0; it < iters; ++it) {
#pragma unroll
        for(int k = 0; k < 8; ++k) {
            const uint32_t addr = base + (uint32_t) (((it * 8 + k) & 31) * 512);
            uint32_t x, y, z, w;
            asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(x), "=r"(y), "=r"(z), "=r"(w) : "r"(addr));
            acc ^= x ^ y ^ z ^ w;
        }
    }
    __syncthreads();
    const unsigned long long c1 = clock64();
    out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
    if(threadIdx.x == 0) atomicMax(cycles, c1 - c0);
}

static int run_lds(msa_ctx *ctx, int iters, msa_op_probe *res)
{
    const int threads = 256;
    int per_sm = 0;
    MSA_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, probe_lds_kernel, threads, 0));
    per_sm = std::min(per_sm, 4);
    const int blocks = ctx->num_sms * per_sm;
    MSA_CUDA_TRY(ctx, ctx->tasks.ensure((size_t) blocks * threads * 4 + 64));
    uint32_t *out = (uint32_t *) ctx->tasks.ptr;
    auto *cyc = (unsigned long long *) (out + (size_t) blocks * threads);
    cudaStream_t s = ctx->stream;
    for(int rep = 0; rep < 2; ++rep) {   // first pass warms up
        MSA_CUDA_TRY(ctx, cudaMemsetAsync(cyc, 0, 8, s));
        MSA_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[0], s));
        probe_lds_kernel<<<blocks, threads, 0, s>>>(out, iters, cyc);
        MSA_CUDA_TRY(ctx, cudaGetLastError());
        MSA_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[1], s));
        ctx->launches++;
    }
    unsigned long long cycles = 0;
    MSA_CUDA_TRY(ctx, cudaMemcpyAsync(&cycles, cyc, 8, cudaMemcpyDeviceToHost, s));
    MSA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    const double bytes_per_sm = (double) per_sm * threads * iters * 8.0 * 16.0;
    res->ops_per_clk_sm = cycles ? bytes_per_sm / (double) cycles : 0.0;
    res->ms = ms;
    res->lane_ops = (uint64_t) ((double) blocks * threads * iters * 8.0);
    res->sm_clock_mhz = ms > 0 ? (double) cycles / (ms * 1e3) : 0.0;
    return MSA_OK;
}

template <int OP>
static int run(msa_ctx *ctx, int iters, msa_op_probe *res)
{
    const int threads = 256;
    int per_sm = 0;
    MSA_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, probe_kernel<OP>, threads, 0));
    per_sm = std::min(per_sm, 4);
    const int blocks = ctx->num_sms * per_sm;
    MSA_CUDA_TRY(ctx, ctx->tasks.ensure((size_t) 4096 * 4 + (size_t) blocks * threads * 4 + 64));
    uint32_t *in = (uint32_t *) ctx->tasks.ptr;
    uint32_t *out = in + 4096;
    auto *cyc = (unsigned long long *) (out + (size_t) blocks * threads);
    cudaStream_t s = ctx->stream;
    MSA_CUDA_TRY(ctx, cudaMemsetAsync(in, 0x5a, 4096 * 4, s));
    for(int rep = 0; rep < 2; ++rep) {   // first pass warms up
        MSA_CUDA_TRY(ctx, cudaMemsetAsync(cyc, 0, 8, s));
        MSA_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[0], s));
        probe_kernel<OP><<<blocks, threads, 0, s>>>(in, out, iters, cyc);
        MSA_CUDA_TRY(ctx, cudaGetLastError());
        MSA_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[1], s));
        ctx->launches++;
    }
    unsigned long long cycles = 0;
    MSA_CUDA_TRY(ctx, cudaMemcpyAsync(&cycles, cyc, 8, cudaMemcpyDeviceToHost, s));
    MSA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    const double lane_ops_per_sm = (double) per_sm * threads * iters * 8.0;
    res->ops_per_clk_sm = cycles ? lane_ops_per_sm / (double) cycles : 0.0;
    res->ms = ms;
    res->lane_ops = (uint64_t) ((double) blocks * threads * iters * 8.0);
    res->sm_clock_mhz = ms > 0 ? (double) cycles / (ms * 1e3) : 0.0;
    return MSA_OK;
}

}  // namespace probe
}  // namespace msa

extern "C" int msa_probe_op(msa_ctx *ctx, int op, int iters, msa_op_probe *out)
{
    if(!ctx || !out || iters <= 0) return MSA_ERR_INVALID;
    cudaSetDevice(ctx->device);
    using namespace msa::probe;
    switch(op) {
        case 0: return run<0>(ctx, iters, out);
        case 1: return run<1>(ctx, iters, out);
        case 2: return run<2>(ctx, iters, out);
        case 3: return run<3>(ctx, iters, out);
        case 4: return run<4>(ctx, iters, out);
        case 5: return run<5>(ctx, iters, out);
        case 6: return run<6>(ctx, iters, out);
        case 7: return run<7>(ctx, iters, out);
        case 8: return run<8>(ctx, iters, out);
        case 9: return run<9>(ctx, iters, out);
        case 10: return run<10>(ctx, iters, out);
        case 11: return run<11>(ctx, iters, out);
        case 12: return run<12>(ctx, iters, out);
        case 13: return run<13>(ctx, iters, out);
        case 14: return run<14>(ctx, iters, out);
        case 15: return run_lds(ctx, iters, out);
        default: return MSA_ERR_INVALID;
    }
}
