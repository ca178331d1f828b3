// Stable LSD radix sort and exclusive scan (see dem_sort.cuh).
#include "dem_sort.cuh"

#include <algorithm>

namespace dem {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr size_t kScanChunk = (size_t)kScanThreads * kScanItems;  // 4096 words
constexpr int kScanTopThreads = 1024;
constexpr int kScanTopItems = 8;
constexpr size_t kScanMaxPartials = (size_t)kScanTopThreads * kScanTopItems;

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Exclusive scan of one value per thread across the block; returns the
// thread's exclusive prefix and writes the block total.
template <int THREADS>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warpTot,
                                                         uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warpTot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        constexpr int W = THREADS / 32;
        uint32_t t = lane < W ? warpTot[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < W) warpTot[lane] = t;  // inclusive over warps
    }
    __syncthreads();
    const uint32_t warpPrefix = warp > 0 ? warpTot[warp - 1] : 0u;
    total = warpTot[THREADS / 32 - 1];
    return warpPrefix + x - v;
}

__global__ void __launch_bounds__(kScanThreads)
scan_reduce_kernel(const uint32_t* __restrict__ data, size_t len, uint32_t* __restrict__ partials) {
    __shared__ uint32_t warpTot[kScanThreads / 32];
    const size_t base = (size_t)blockIdx.x * kScanChunk;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        size_t i = base + (size_t)k * kScanThreads + threadIdx.x;
        if (i < len) s += data[i];
    }
    uint32_t total;
    (void)block_exclusive_scan<kScanThreads>(s, warpTot, total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanTopThreads)
scan_partials_kernel(uint32_t* __restrict__ partials, uint32_t np) {
    __shared__ uint32_t warpTot[kScanTopThreads / 32];
    uint32_t v[kScanTopItems];
    uint32_t s = 0;
    const uint32_t b = threadIdx.x * kScanTopItems;
#pragma unroll
    for (int k = 0; k < kScanTopItems; ++k) {
        v[k] = (b + k < np) ? partials[b + k] : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t run = block_exclusive_scan<kScanTopThreads>(s, warpTot, total);
#pragma unroll
    for (int k = 0; k < kScanTopItems; ++k) {
        if (b + k < np) partials[b + k] = run;
        run += v[k];
    }
}

__global__ void __launch_bounds__(kScanThreads)
scan_apply_kernel(uint32_t* __restrict__ data, size_t len, const uint32_t* __restrict__ partials) {
    __shared__ uint32_t warpTot[kScanThreads / 32];
    const size_t base = (size_t)blockIdx.x * kScanChunk + (size_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < len) ? data[base + k] : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t run = block_exclusive_scan<kScanThreads>(s, warpTot, total) + partials[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < len) data[base + k] = run;
        run += v[k];
    }
}

// Per-tile digit counts, written digit-major: hist[d * numTiles + tile].
template <int BITS>
__global__ void __launch_bounds__(kSortThreads)
upsweep_kernel(const uint32_t* __restrict__ keys, uint32_t n, int shift, uint32_t rows,
               uint32_t* __restrict__ hist, uint32_t numTiles) {
    constexpr int R = 1 << BITS;
    __shared__ uint32_t h[R];
    for (int d = threadIdx.x; d < R; d += kSortThreads) h[d] = 0;
    __syncthreads();
    const uint32_t mask = rows - 1u;
    const int lane = threadIdx.x & 31;
    const size_t base = (size_t)blockIdx.x * kSortTile;
#pragma unroll 4
    for (int k = 0; k < kSortItems; ++k) {
        const size_t idx = base + (size_t)k * kSortThreads + threadIdx.x;
        const bool valid = idx < n;
        const uint32_t d = valid ? ((__ldg(keys + idx) >> shift) & mask) : 0xffffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (valid && (__ffs(peers) - 1) == lane) atomicAdd(&h[d], (uint32_t)__popc(peers));
    }
    __syncthreads();
    for (uint32_t d = threadIdx.x; d < rows; d += kSortThreads)
        hist[(size_t)d * numTiles + blockIdx.x] = h[d];
}

// Stable scatter.  Warp w of the tile owns the contiguous run of 512 keys
// [w*512, (w+1)*512); it walks them 32 at a time in index order and ranks
// equal digits with match_any, so ranks follow the input order inside the
// warp; warps are then offset by the counts of lower warps, and tiles by the
// scanned digit-major table.  Stability follows.
template <int BITS, bool IDENT>
__global__ void __launch_bounds__(kSortThreads)
downsweep_kernel(const uint32_t* __restrict__ keysIn, const uint32_t* __restrict__ valsIn,
                 uint32_t* __restrict__ keysOut, uint32_t* __restrict__ valsOut, uint32_t n,
                 int shift, uint32_t rows, const uint32_t* __restrict__ hist, uint32_t numTiles) {
    constexpr int R = 1 << BITS;
    __shared__ uint16_t cnt[kSortWarps][R];
    __shared__ uint32_t gbase[R];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t mask = rows - 1u;
    uint16_t* flat = &cnt[0][0];
    for (int i = threadIdx.x; i < kSortWarps * R; i += kSortThreads) flat[i] = 0;
    for (uint32_t d = threadIdx.x; d < rows; d += kSortThreads)
        gbase[d] = hist[(size_t)d * numTiles + blockIdx.x];
    __syncthreads();

    const size_t wbase = (size_t)blockIdx.x * kSortTile + (size_t)warp * (kSortItems * 32);
    uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const size_t idx = wbase + (size_t)k * 32 + lane;
        const bool valid = idx < n;
        key[k] = valid ? __ldg(keysIn + idx) : 0u;
        if (IDENT) val[k] = (uint32_t)idx;
        else val[k] = valid ? __ldg(valsIn + idx) : 0u;
    }
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const size_t idx = wbase + (size_t)k * 32 + lane;
        const bool valid = idx < n;
        const uint32_t d = valid ? ((key[k] >> shift) & mask) : 0xffffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t c = valid ? (uint32_t)cnt[warp][d] : 0u;
        __syncwarp();
        if (valid && (peers & lt) == 0u) cnt[warp][d] = (uint16_t)(c + (uint32_t)__popc(peers));
        __syncwarp();
        rank[k] = c + (uint32_t)__popc(peers & lt);
    }
    __syncthreads();
    for (uint32_t d = threadIdx.x; d < rows; d += kSortThreads) {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = cnt[w][d];
            cnt[w][d] = (uint16_t)run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const size_t idx = wbase + (size_t)k * 32 + lane;
        if (idx < n) {
            const uint32_t d = (key[k] >> shift) & mask;
            const uint32_t dst = gbase[d] + (uint32_t)cnt[warp][d] + rank[k];
            keysOut[dst] = key[k];
            valsOut[dst] = val[k];
        }
    }
}

__global__ void iota_kernel(uint32_t* __restrict__ v, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

template <int BITS>
cudaError_t run_pass(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout,
                     uint32_t n, int shift, int bits, bool ident, uint32_t* hist,
                     uint32_t* partials, cudaStream_t st, int* launches) {
    const uint32_t numTiles = (n + kSortTile - 1) / kSortTile;
    const uint32_t rows = 1u << bits;
    upsweep_kernel<BITS><<<numTiles, kSortThreads, 0, st>>>(kin, n, shift, rows, hist, numTiles);
    if (launches) ++*launches;
    cudaError_t e = exclusive_scan_u32(hist, (size_t)rows * numTiles, partials, st, launches);
    if (e != cudaSuccess) return e;
    if (ident)
        downsweep_kernel<BITS, true><<<numTiles, kSortThreads, 0, st>>>(kin, vin, kout, vout, n,
                                                                        shift, rows, hist, numTiles);
    else
        downsweep_kernel<BITS, false><<<numTiles, kSortThreads, 0, st>>>(kin, vin, kout, vout, n,
                                                                         shift, rows, hist, numTiles);
    if (launches) ++*launches;
    return cudaGetLastError();
}

inline size_t align256(size_t b) { return (b + 255u) & ~(size_t)255u; }

}  // namespace

SortPlan make_sort_plan(uint32_t keyBits) {
    SortPlan p;
    if (keyBits == 0) return p;
    if (keyBits > 32) keyBits = 32;
    p.passes = (int)((keyBits + 10u) / 11u);
    const int per = (int)((keyBits + (uint32_t)p.passes - 1u) / (uint32_t)p.passes);
    int shift = 0;
    for (int i = 0; i < p.passes; ++i) {
        p.shift[i] = shift;
        p.bits[i] = std::min(per, (int)keyBits - shift);
        shift += per;
    }
    p.radixBits = per <= 6 ? 6 : per <= 8 ? 8 : per <= 10 ? 10 : 11;
    return p;
}

size_t sort_hist_words(uint32_t n, const SortPlan& plan) {
    const size_t numTiles = (n + kSortTile - 1) / kSortTile;
    int maxBits = 0;
    for (int i = 0; i < plan.passes; ++i) maxBits = std::max(maxBits, plan.bits[i]);
    return numTiles * ((size_t)1 << maxBits);
}

size_t sort_scan_partials(size_t words) {
    return std::max<size_t>(1, (words + kScanChunk - 1) / kScanChunk);
}

size_t sort_scratch_bytes(uint32_t n, uint32_t keyBits) {
    const SortPlan plan = make_sort_plan(keyBits);
    const size_t hw = sort_hist_words(n, plan);
    return 2 * align256(sizeof(uint32_t) * std::max<size_t>(n, 1)) +
           align256(sizeof(uint32_t) * std::max<size_t>(hw, 1)) +
           align256(sizeof(uint32_t) * sort_scan_partials(hw));
}

SortScratch carve_sort_scratch(void* base, uint32_t n, uint32_t keyBits) {
    const SortPlan plan = make_sort_plan(keyBits);
    const size_t hw = sort_hist_words(n, plan);
    char* p = static_cast<char*>(base);
    SortScratch s;
    s.altKeys = reinterpret_cast<uint32_t*>(p);
    p += align256(sizeof(uint32_t) * std::max<size_t>(n, 1));
    s.altVals = reinterpret_cast<uint32_t*>(p);
    p += align256(sizeof(uint32_t) * std::max<size_t>(n, 1));
    s.hist = reinterpret_cast<uint32_t*>(p);
    p += align256(sizeof(uint32_t) * std::max<size_t>(hw, 1));
    s.partials = reinterpret_cast<uint32_t*>(p);
    return s;
}

cudaError_t exclusive_scan_u32(uint32_t* data, size_t len, uint32_t* partials, cudaStream_t st,
                               int* launches) {
    if (len == 0) return cudaSuccess;
    const size_t nb = (len + kScanChunk - 1) / kScanChunk;
    if (nb > kScanMaxPartials) return cudaErrorInvalidValue;
    scan_reduce_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(data, len, partials);
    scan_partials_kernel<<<1, kScanTopThreads, 0, st>>>(partials, (uint32_t)nb);
    scan_apply_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(data, len, partials);
    if (launches) *launches += 3;
    return cudaGetLastError();
}

cudaError_t radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t keyBits,
                             bool identityVals, const SortScratch& s, cudaStream_t st,
                             uint32_t** keysOut, uint32_t** valsOut, int* launches) {
    *keysOut = keys;
    *valsOut = vals;
    if (n == 0) return cudaSuccess;
    const SortPlan plan = make_sort_plan(keyBits);
    if (plan.passes == 0) {
        if (identityVals) {
            iota_kernel<<<(n + 255) / 256, 256, 0, st>>>(vals, n);
            if (launches) ++*launches;
        }
        return cudaGetLastError();
    }
    if (sort_scan_partials(sort_hist_words(n, plan)) > kScanMaxPartials)
        return cudaErrorInvalidValue;
    uint32_t *ki = keys, *vi = vals, *ko = s.altKeys, *vo = s.altVals;
    for (int p = 0; p < plan.passes; ++p) {
        const bool ident = identityVals && p == 0;
        cudaError_t e;
        switch (plan.radixBits) {
            case 6:
                e = run_pass<6>(ki, vi, ko, vo, n, plan.shift[p], plan.bits[p], ident, s.hist,
                                s.partials, st, launches);
                break;
            case 8:
                e = run_pass<8>(ki, vi, ko, vo, n, plan.shift[p], plan.bits[p], ident, s.hist,
                                s.partials, st, launches);
                break;
            case 10:
                e = run_pass<10>(ki, vi, ko, vo, n, plan.shift[p], plan.bits[p], ident, s.hist,
                                 s.partials, st, launches);
                break;
            default:
                e = run_pass<11>(ki, vi, ko, vo, n, plan.shift[p], plan.bits[p], ident, s.hist,
                                 s.partials, st, launches);
                break;
        }
        if (e != cudaSuccess) return e;
        std::swap(ki, ko);
        std::swap(vi, vo);
    }
    *keysOut = ki;
    *valsOut = vi;
    return cudaSuccess;
}

}  // namespace dem
