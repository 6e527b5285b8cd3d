// msa_nw_all_pairs_noalloc: all-pairs Needleman-Wunsch that allocates no
// memory of any kind on the device.
//
// Who needs it: callers that are not allowed to call cudaMalloc at the point
// where they score sequences, e.g. a host runtime whose device memory is all
// owned by its own pool and that forbids allocations after start-up, code that
// must not trigger the implicit device synchronisation an allocation can cause,
// or a latency-critical loop that cannot afford one. They pass sequences and
// the output already in device memory; everything else the kernel needs lives
// in one fixed, file-scope device array owned by this library.
//
// The scratch array holds, per call: an error flag (cleared at the start of
// every call), the sequence offsets and lengths (copied in by every call), and
// one strip-boundary row per resident warp. Every call on a device shares that
// one array and it keeps the last call's contents, so calls that overlap on the
// GPU (two host threads, or two streams, using the same device at the same
// time) race with each other and must be serialised by the caller.
//
// Limits (checked, MSA_ERR_TOO_LARGE otherwise): n <= kMaxSeqs sequences, and
// every sequence short enough that one 4-warp block's boundary rows fit the
// scratch (about one million units).
#include <algorithm>
#include <cstring>
#include <mutex>

#include "msa_internal.hpp"

namespace msa {
namespace noalloc {

constexpr size_t kScratchBytes = size_t(16) << 20;       // 16 MiB per device
constexpr uint32_t kMaxSeqs = 65536;
constexpr int kR = 16;                                   // rows per lane
constexpr int kSH = 32 * kR;                             // rows per strip
constexpr int kWPB = 4;                                  // warps per block
constexpr size_t kHeaderWords = 64;
constexpr size_t kMetaWords = size_t(kMaxSeqs) * 4;      // offs and lens, 2 x u64 each

// The scratch. In host code this symbol is only a stand-in: the device address
// comes from cudaGetSymbolAddress (scratch_for_device below).
static __device__ __align__(256) uint32_t g_scratch[kScratchBytes / 4];

constexpr unsigned kFull = 0xffffffffu;

struct Params {
    const uint8_t *units;
    uint32_t n;
    int32_t g;
    int32_t *out;
    uint64_t stride;      // boundary-row words per warp
    int gap_invalid;      // some GAP entry of the table lies outside the reference's storage
    int8_t ext[26 * 26];  // score for units x, y as the reference reads them
};

template <int K>
__device__ __forceinline__ int32_t sbyte(uint32_t w)
{
    int32_t r;
    asm("prmt.b32 %0, %1, 0, %2;" : "=r"(r) : "r"(w), "n"((K) | ((K | 8) << 4) | ((K | 8) << 8) | ((K | 8) << 12)));
    return r;
}

__device__ __forceinline__ uint32_t unit_at(const uint8_t *s, uint64_t len, int64_t k)
{
    return (k >= 0 && (uint64_t) k < len) ? s[k] : (uint32_t) MSA_UNIT_END;
}

// One pair on the calling warp, with the reference's semantics: rows stop at
// the first END unit, END columns copy their left neighbour, the padded column
// width is swept (src/pairwise/needleman/impl/sequential.cpp:29-68).
__device__ void score_pair(const Params &p, const uint8_t *rows, uint64_t lr, const uint8_t *cols, uint64_t lc,
                           int8_t *sprof, const int8_t *stab, uint32_t *bound, int lane, int32_t &result)
{
    const int plen_r = (int) ((lr + 2) / 3 * 3), ncols = (int) ((lc + 2) / 3 * 3);
    // Effective rows: up to the first END unit.
    int nrows = plen_r;
    for(int base = 0; base < plen_r; base += 32) {
        const uint32_t u = unit_at(rows, lr, base + lane);
        const unsigned m = __ballot_sync(kFull, u == MSA_UNIT_END && base + lane < plen_r);
        if(m) { nrows = base + __ffs(m) - 1; break; }
    }
    if(nrows == 0) { result = -ncols * p.g; return; }
    if(ncols == 0) { result = -nrows * p.g; return; }

    const int nstrips = (nrows + kSH - 1) / kSH;
    for(int s = 0; s < nstrips; ++s) {
        const int i0 = s * kSH;
        const bool first = s == 0, last = s == nstrips - 1;
        const int rl = nrows - 1 - i0;
        const int klast = last ? rl / kR : 31, rlast = rl % kR;

        // Stage this lane's profile bytes [code][lane][kR] from the table.
        __syncwarp();
        uint32_t xr[kR];
#pragma unroll
        for(int r = 0; r < kR; ++r) {
            const int row = i0 + lane * kR + r;
            xr[r] = row < nrows ? unit_at(rows, lr, row) : 0u;
        }
        for(int b = 0; b < 26; ++b) {
            uint32_t w[kR / 4];
#pragma unroll
            for(int q = 0; q < kR / 4; ++q) {
                w[q] = 0;
#pragma unroll
                for(int k = 0; k < 4; ++k) {
                    const uint32_t x = xr[4 * q + k];
                    // Entries outside the reference's storage all involve
                    // the GAP unit; the kernel's GAP rule has already flagged
                    // any call that could read one (they stage as 0).
                    const int idx = (int) x * 26 + b;
                    w[q] |= ((uint32_t) (uint8_t) stab[idx]) << (8 * k);
                }
            }
            *reinterpret_cast<uint4 *>(sprof + b * kSH + lane * kR) = make_uint4(w[0], w[1], w[2], w[3]);
        }
        __syncwarp();

        int32_t H[kR];
#pragma unroll
        for(int r = 0; r < kR; ++r) H[r] = -(i0 + lane * kR + r + 1) * p.g;
        int32_t diag = -(i0 + lane * kR) * p.g;
        int32_t hlast = H[kR - 1];
        const int tend = ncols + klast;
        for(int t = 0; t < tend; ++t) {
            int32_t up = __shfl_up_sync(kFull, hlast, 1);
            const int j = t - lane;
            if(lane == 0) up = first ? -(t + 1) * p.g : (int32_t) bound[min(t, ncols - 1)];
            if(j >= 0 && j < ncols) {
                const uint32_t b = unit_at(cols, lc, j);
                if(b != MSA_UNIT_END) {
                    const uint4 pw = *reinterpret_cast<const uint4 *>(sprof + b * kSH + lane * kR);
                    const uint32_t wv[4] = {pw.x, pw.y, pw.z, pw.w};
                    int32_t d = diag, u = up;
#pragma unroll
                    for(int q = 0; q < 4; ++q) {
#pragma unroll
                        for(int k = 0; k < 4; ++k) {
                            const int r = 4 * q + k;
                            const int32_t sc = k == 0 ? sbyte<0>(wv[q]) : k == 1 ? sbyte<1>(wv[q])
                                             : k == 2 ? sbyte<2>(wv[q]) : sbyte<3>(wv[q]);
                            const int32_t h = __viaddmax_s32(u, -p.g, __viaddmax_s32(H[r], -p.g, d + sc));
                            d = H[r];
                            H[r] = h;
                            u = h;
                        }
                    }
                }
                hlast = H[kR - 1];
                if(!last && lane == 31) bound[j] = (uint32_t) hlast;
                if(last && lane == klast && j == ncols - 1) {
                    int32_t v = H[0];
#pragma unroll
                    for(int r = 1; r < kR; ++r) if(r == rlast) v = H[r];
                    result = v;
                }
                diag = up;
            }
        }
        __syncwarp();
        if(last) result = __shfl_sync(kFull, result, klast);
    }
}

constexpr size_t kSmem = (size_t) kWPB * 26 * kSH;

__global__ void __launch_bounds__(kWPB * 32) noalloc_kernel(Params p, uint32_t *scratch)
{
    extern __shared__ __align__(16) int8_t sprof_all[];
    __shared__ int8_t stab[26 * 26];
    for(int i = threadIdx.x; i < 26 * 26; i += blockDim.x) stab[i] = p.ext[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t *err = scratch;
    const uint64_t *offs = reinterpret_cast<const uint64_t *>(scratch + kHeaderWords);
    const uint64_t *lens = offs + kMaxSeqs;
    const uint64_t gw = (uint64_t) blockIdx.x * kWPB + warp;
    const uint64_t nw = (uint64_t) gridDim.x * kWPB;
    uint32_t *bound = scratch + kHeaderWords + kMetaWords + gw * p.stride;
    // msa_nw_all_pairs's rule: with such a table, a GAP unit anywhere in any
    // sequence makes the whole call undefined, wherever the pairs would read it.
    if(p.gap_invalid) {
        for(uint64_t q = gw; q < p.n; q += nw) {
            const uint8_t *u = p.units + offs[q];
            bool gap = false;
            for(uint64_t k = lane; k < lens[q]; k += 32) gap |= u[k] == MSA_UNIT_GAP;
            if(__any_sync(kFull, gap) && lane == 0) atomicOr(err, 1u);
        }
    }
    const uint64_t total = (uint64_t) p.n * (p.n - 1) / 2;
    for(uint64_t k = gw; k < total; k += nw) {
        // k = i(i-1)/2 + j, i > j (src/pairwise/pairwise.cpp:73-85).
        uint64_t i = (uint64_t) ((1.0 + sqrt(1.0 + 8.0 * (double) k)) * 0.5);
        while(i * (i - 1) / 2 > k) --i;
        while((i + 1) * i / 2 <= k) ++i;
        const uint64_t j = k - i * (i - 1) / 2;
        const uint64_t bi = (lens[i] + 2) / 3, bj = (lens[j] + 2) / 3;
        const uint64_t r = bi > bj ? i : j, c = bi > bj ? j : i;   // sequential.cpp:87-91
        int32_t res = 0;
        score_pair(p, p.units + offs[r], lens[r], p.units + offs[c], lens[c], sprof_all + warp * 26 * kSH, stab, bound,
                   lane, res);
        if(lane == 0) p.out[k] = res;
    }
}

// Device address of the scratch array for each device, looked up once per
// device with that device current (the first call on a device does it, so
// that first call should come before any stream capture). The kernel's
// dynamic shared-memory limit is raised at the same time.
static std::mutex g_lock;
static void *g_addr[64];
static bool g_ready[64];

static int scratch_for_device(int dev, void **out, std::string *err)
{
    if(dev < 0 || dev >= 64) { *err = "device index out of range"; return MSA_ERR_INVALID; }
    std::lock_guard<std::mutex> lk(g_lock);
    if(!g_ready[dev]) {
        void *ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
        if(e != cudaSuccess || ptr == nullptr) {
            cudaGetLastError();
            *err = std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
            return MSA_ERR_CUDA;
        }
        const cudaError_t e2 = cudaFuncSetAttribute(noalloc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) kSmem);
        if(e2 != cudaSuccess) {
            cudaGetLastError();
            *err = std::string("cudaFuncSetAttribute failed: ") + cudaGetErrorString(e2);
            return MSA_ERR_CUDA;
        }
        g_addr[dev] = ptr;
        g_ready[dev] = true;
    }
    *out = g_addr[dev];
    return MSA_OK;
}

static thread_local std::string g_err;

}  // namespace noalloc
}  // namespace msa

extern "C" const char *msa_noalloc_last_error(void) { return msa::noalloc::g_err.c_str(); }

extern "C" int msa_nw_all_pairs_noalloc(const uint8_t *units, const uint64_t *offs, const uint64_t *lens,
                                        uint32_t n, const msa_table *table, int32_t *out, void *stream)
{
    using namespace msa::noalloc;
    std::string &err = g_err;
    err.clear();
    if(!table || (n && (!offs || !lens))) return MSA_ERR_INVALID;
    if(n < 2) return MSA_OK;
    if(!units || !out) return MSA_ERR_INVALID;
    if(n > kMaxSeqs) { err = "more than 65536 sequences"; return MSA_ERR_TOO_LARGE; }
    msa::ExtTable ext;
    int rc = msa::make_ext_table(table, &ext, &err);
    if(rc) return rc;
    uint64_t maxlen = 0;
    for(uint32_t i = 0; i < n; ++i) maxlen = std::max<uint64_t>(maxlen, lens[i]);
    const int64_t vb = (int64_t) (2 * (maxlen + 3) + 2) * std::max<int64_t>(ext.max_abs, ext.penalty);
    if(vb >= (1ll << 30)) { err = "scores could exceed the int32 range"; return MSA_ERR_TOO_LARGE; }
    const uint64_t stride = msa::round_up(maxlen + 8, 32);
    const uint64_t avail = kScratchBytes / 4 - kHeaderWords - kMetaWords;
    if(stride * kWPB > avail) { err = "a sequence is too long for the fixed scratch (about 1M units)"; return MSA_ERR_TOO_LARGE; }

    int dev = 0;
    if(cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return MSA_ERR_NO_DEVICE; }
    void *base = nullptr;
    rc = scratch_for_device(dev, &base, &err);
    if(rc) return rc;
    uint32_t *scratch = static_cast<uint32_t *>(base);
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    Params p{};
    p.units = units;
    p.n = n;
    p.g = ext.penalty;
    p.out = out;
    p.stride = stride;
    for(int x = 0; x < 26; ++x)
        for(int y = 0; y < 26; ++y)
            if((x == MSA_UNIT_GAP || y == MSA_UNIT_GAP) && x != MSA_UNIT_END && y != MSA_UNIT_END &&
               !ext.valid[x * 26 + y])
                p.gap_invalid = 1;
    std::memcpy(p.ext, ext.score, sizeof(p.ext));

    int sms = 0, bps = 0;
    if(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
       cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, noalloc_kernel, kWPB * 32, kSmem) != cudaSuccess || bps < 1) {
        cudaGetLastError();
        err = "device query failed";
        return MSA_ERR_CUDA;
    }
    const uint64_t total = (uint64_t) n * (n - 1) / 2;
    uint64_t blocks = std::min<uint64_t>((uint64_t) sms * bps, avail / (stride * kWPB));
    blocks = std::max<uint64_t>(1, std::min<uint64_t>(blocks, (total + kWPB - 1) / kWPB));

    // Clear the error flag; copy offsets and lengths in (the array keeps the
    // previous call's contents otherwise).
    cudaError_t e = cudaMemsetAsync(scratch, 0, kHeaderWords * 4, s);
    if(!e) e = cudaMemcpyAsync(scratch + kHeaderWords, offs, n * sizeof(uint64_t), cudaMemcpyHostToDevice, s);
    if(!e) e = cudaMemcpyAsync(scratch + kHeaderWords + 2 * (size_t) kMaxSeqs, lens, n * sizeof(uint64_t),
                               cudaMemcpyHostToDevice, s);
    if(e) { cudaGetLastError(); err = cudaGetErrorString(e); return MSA_ERR_CUDA; }
    noalloc_kernel<<<(unsigned) blocks, kWPB * 32, kSmem, s>>>(p, scratch);
    e = cudaGetLastError();
    if(e) { err = cudaGetErrorString(e); return MSA_ERR_CUDA; }
    uint32_t flag = 0;
    e = cudaMemcpyAsync(&flag, scratch, sizeof(flag), cudaMemcpyDeviceToHost, s);
    if(!e) e = cudaStreamSynchronize(s);
    if(e) { cudaGetLastError(); err = cudaGetErrorString(e); return MSA_ERR_CUDA; }
    if(flag) { err = "GAP unit with this table reads past the reference's table storage"; return MSA_ERR_UNDEFINED; }
    return MSA_OK;
}
