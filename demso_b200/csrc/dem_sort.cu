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

// ---------------------------------------------------------------- onesweep
constexpr uint32_t kFlagAgg = 1u << 30;   // tile aggregate published
constexpr uint32_t kFlagIncl = 2u << 30;  // inclusive prefix published
constexpr uint32_t kValueMask = (1u << 30) - 1u;
constexpr int kHistBlocksPerSM = 2;

// Global digit histograms of every pass.  Each thread walks a run of
// consecutive keys and adds one count per run of equal digits, so nearly
// sorted input (the step's common case) needs few shared-memory atomics.
template <int BITS>
__global__ void __launch_bounds__(kSortThreads)
global_hist_kernel(const uint32_t* __restrict__ keys, uint32_t n, int passes, int4 shifts,
                   int4 rowsv, uint32_t* __restrict__ gh) {
    constexpr int R = 1 << BITS;
    __shared__ uint32_t h[4][R];
    const int sh[4] = {shifts.x, shifts.y, shifts.z, shifts.w};
    const int rw[4] = {rowsv.x, rowsv.y, rowsv.z, rowsv.w};
    for (int i = threadIdx.x; i < 4 * R; i += kSortThreads) (&h[0][0])[i] = 0;
    __syncthreads();
    const uint32_t per = 16;
    const size_t stride = (size_t)gridDim.x * kSortThreads * per;
    for (size_t base = ((size_t)blockIdx.x * kSortThreads + threadIdx.x) * per; base < n;
         base += stride) {
        const uint32_t cnt = (uint32_t)min((size_t)per, (size_t)n - base);
        for (int p = 0; p < passes; ++p) {
            const uint32_t mask = (uint32_t)rw[p] - 1u;
            uint32_t cur = (__ldg(keys + base) >> sh[p]) & mask, run = 1;
            for (uint32_t k = 1; k < cnt; ++k) {
                const uint32_t d = (__ldg(keys + base + k) >> sh[p]) & mask;
                if (d == cur) {
                    ++run;
                } else {
                    atomicAdd(&h[p][cur], run);
                    cur = d;
                    run = 1;
                }
            }
            atomicAdd(&h[p][cur], run);
        }
    }
    __syncthreads();
    for (int p = 0; p < passes; ++p)
        for (int d = threadIdx.x; d < rw[p]; d += kSortThreads)
            if (h[p][d]) atomicAdd(gh + (size_t)p * R + d, h[p][d]);
}

// Exclusive scan of each pass's row of the global histogram (one block per pass).
template <int BITS>
__global__ void __launch_bounds__(1024) global_hist_scan_kernel(uint32_t* __restrict__ gh) {
    constexpr int R = 1 << BITS;
    constexpr int PER = (R + 1023) / 1024;
    __shared__ uint32_t warpTot[32];
    uint32_t* row = gh + (size_t)blockIdx.x * R;
    uint32_t v[PER];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int d = threadIdx.x * PER + k;
        v[k] = d < R ? row[d] : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t run = block_exclusive_scan<1024>(s, warpTot, total);
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int d = threadIdx.x * PER + k;
        if (d < R) row[d] = run;
        run += v[k];
    }
}

template <int BITS, bool IDENT>
__global__ void __launch_bounds__(kSortThreads, 3)
onesweep_kernel(const uint32_t* __restrict__ keysIn, const uint32_t* __restrict__ valsIn,
                uint32_t* __restrict__ keysOut, uint32_t* __restrict__ valsOut, uint32_t n,
                int shift, uint32_t rows, const uint32_t* __restrict__ gOffset,
                uint32_t* __restrict__ lookback, uint32_t* __restrict__ errFlag,
                uint32_t holdTile, uint32_t spinLimit) {
    constexpr int R = 1 << BITS;
    __shared__ uint16_t cnt[kSortWarps][R];
    __shared__ uint32_t dbase[R];
    __shared__ uint32_t tileS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t mask = rows - 1u;
    if (threadIdx.x == 0) tileS = atomicAdd(lookback, 1u);
    uint16_t* flat = &cnt[0][0];
    for (int i = threadIdx.x; i < kSortWarps * R; i += kSortThreads) flat[i] = 0;
    __syncthreads();
    const uint32_t tile = tileS;
    volatile uint32_t* lb = lookback + 64;

    const size_t wbase = (size_t)tile * kSortTile + (size_t)warp * (kSortItems * 32);
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
    // per digit: exclusive offsets of the warps and the tile's count, which is
    // published at once (inclusive for tile 0) before any look-back starts
    for (uint32_t d = threadIdx.x; d < rows; d += kSortThreads) {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = cnt[w][d];
            cnt[w][d] = (uint16_t)run;
            run += c;
        }
        if (tile != holdTile) lb[(size_t)tile * rows + d] = (tile == 0 ? kFlagIncl : kFlagAgg) | run;
        dbase[d] = run;
    }
    // decoupled look-back: the tile's exclusive prefix of each digit
    for (uint32_t d = threadIdx.x; d < rows; d += kSortThreads) {
        const uint32_t run = dbase[d];
        uint32_t excl = 0;
        if (tile > 0) {
            uint32_t spins = 0;
            int t = (int)tile - 1;
            while (true) {
                const uint32_t v = lb[(size_t)t * rows + d];
                if ((v & ~kValueMask) == 0u) {
                    if (++spins > spinLimit) {
                        atomicOr(errFlag, kSortTimeoutBit);
                        break;
                    }
                    if (spins > 64) __nanosleep(64);
                    continue;
                }
                excl += v & kValueMask;
                if ((v & kFlagIncl) || t == 0) break;
                --t;
            }
            if (tile != holdTile) lb[(size_t)tile * rows + d] = kFlagIncl | (excl + run);
        }
        dbase[d] = gOffset[d] + excl;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const size_t idx = wbase + (size_t)k * 32 + lane;
        if (idx < n) {
            const uint32_t d = (key[k] >> shift) & mask;
            const uint32_t dst = dbase[d] + (uint32_t)cnt[warp][d] + rank[k];
            if (dst < n) {
                keysOut[dst] = key[k];
                valsOut[dst] = val[k];
            }
        }
    }
}

__global__ void fill_words_kernel(uint32_t* __restrict__ p, uint32_t value, size_t count) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (size_t)gridDim.x * blockDim.x)
        p[i] = value;
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

size_t onesweep_scratch_bytes(uint32_t n, uint32_t keyBits) {
    const SortPlan plan = make_sort_plan(keyBits);
    const size_t numTiles = (n + kSortTile - 1) / kSortTile;
    const size_t R = (size_t)1 << (plan.radixBits ? plan.radixBits : 6);
    return 2 * align256(sizeof(uint32_t) * std::max<size_t>(n, 1)) +
           align256(sizeof(uint32_t) * 4 * R) +
           align256(sizeof(uint32_t) * (64 + numTiles * R));
}

OnesweepScratch carve_onesweep_scratch(void* base, uint32_t n, uint32_t keyBits) {
    const SortPlan plan = make_sort_plan(keyBits);
    const size_t R = (size_t)1 << (plan.radixBits ? plan.radixBits : 6);
    char* p = static_cast<char*>(base);
    OnesweepScratch s;
    s.altKeys = reinterpret_cast<uint32_t*>(p);
    p += align256(sizeof(uint32_t) * std::max<size_t>(n, 1));
    s.altVals = reinterpret_cast<uint32_t*>(p);
    p += align256(sizeof(uint32_t) * std::max<size_t>(n, 1));
    s.globalHist = reinterpret_cast<uint32_t*>(p);
    p += align256(sizeof(uint32_t) * 4 * R);
    s.lookback = reinterpret_cast<uint32_t*>(p);
    return s;
}

namespace {
template <int BITS>
cudaError_t onesweep_impl(uint32_t* keys, uint32_t* vals, uint32_t n, const SortPlan& plan,
                          bool identityVals, const OnesweepScratch& s, uint32_t* errFlag,
                          cudaStream_t st, uint32_t** keysOut, uint32_t** valsOut,
                          int* launches) {
    constexpr int R = 1 << BITS;
    const uint32_t numTiles = (n + kSortTile - 1) / kSortTile;
    // clearing by kernel (not memset nodes) keeps this path valid inside a
    // conditional graph body
    fill_words_kernel<<<4, 256, 0, st>>>(s.globalHist, 0u, 4 * (size_t)R);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t perBlock = (size_t)kSortThreads * 16;
    const unsigned hb = (unsigned)std::max<size_t>(
        1, std::min<size_t>((size_t)sms * kHistBlocksPerSM, (n + perBlock - 1) / perBlock));
    const int4 shifts = make_int4(plan.shift[0], plan.shift[1], plan.shift[2], plan.shift[3]);
    const int4 rowsv = make_int4(1 << plan.bits[0], 1 << plan.bits[1], 1 << plan.bits[2],
                                 1 << plan.bits[3]);
    global_hist_kernel<BITS><<<hb, kSortThreads, 0, st>>>(keys, n, plan.passes, shifts, rowsv,
                                                          s.globalHist);
    global_hist_scan_kernel<BITS><<<plan.passes, 1024, 0, st>>>(s.globalHist);
    if (launches) *launches += 3;
    uint32_t *ki = keys, *vi = vals, *ko = s.altKeys, *vo = s.altVals;
    for (int p = 0; p < plan.passes; ++p) {
        const uint32_t rows = 1u << plan.bits[p];
        const size_t lbWords = 64 + (size_t)numTiles * rows;
        fill_words_kernel<<<(unsigned)std::min<size_t>((lbWords + 255) / 256, 1184), 256, 0, st>>>(
            s.lookback, 0u, lbWords);
        if (launches) ++*launches;
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        const uint32_t* go = s.globalHist + (size_t)p * R;
        if (identityVals && p == 0)
            onesweep_kernel<BITS, true><<<numTiles, kSortThreads, 0, st>>>(
                ki, vi, ko, vo, n, plan.shift[p], rows, go, s.lookback, errFlag, s.holdTile,
                s.spinLimit);
        else
            onesweep_kernel<BITS, false><<<numTiles, kSortThreads, 0, st>>>(
                ki, vi, ko, vo, n, plan.shift[p], rows, go, s.lookback, errFlag, s.holdTile,
                s.spinLimit);
        if (launches) ++*launches;
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        std::swap(ki, ko);
        std::swap(vi, vo);
    }
    *keysOut = ki;
    *valsOut = vi;
    return cudaSuccess;
}
}  // namespace

cudaError_t onesweep_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t keyBits,
                                bool identityVals, const OnesweepScratch& s, uint32_t* errFlag,
                                cudaStream_t st, uint32_t** keysOut, uint32_t** valsOut,
                                int* launches) {
    *keysOut = keys;
    *valsOut = vals;
    if (n == 0) return cudaSuccess;
    if (n >= (1u << 30)) return cudaErrorInvalidValue;
    const SortPlan plan = make_sort_plan(keyBits);
    if (plan.passes == 0) {
        if (identityVals) {
            iota_kernel<<<(n + 255) / 256, 256, 0, st>>>(vals, n);
            if (launches) ++*launches;
        }
        return cudaGetLastError();
    }
    switch (plan.radixBits) {
        case 6:
            return onesweep_impl<6>(keys, vals, n, plan, identityVals, s, errFlag, st, keysOut,
                                    valsOut, launches);
        case 8:
            return onesweep_impl<8>(keys, vals, n, plan, identityVals, s, errFlag, st, keysOut,
                                    valsOut, launches);
        case 10:
            return onesweep_impl<10>(keys, vals, n, plan, identityVals, s, errFlag, st, keysOut,
                                     valsOut, launches);
        default:
            return onesweep_impl<11>(keys, vals, n, plan, identityVals, s, errFlag, st, keysOut,
                                     valsOut, launches);
    }
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
