// Incremental stable sort of the context step (see dem_incsort.cuh).
#include "dem_incsort.cuh"

#include <algorithm>

namespace dem {
namespace {

constexpr int kThreads = 256;
constexpr uint32_t kMinCellItems = 2;
// scan blocks at most: a block of cells_apply sums the totals of the blocks
// below it, at most kMaxScanBlocks / kThreads loads a thread
constexpr uint32_t kMaxScanBlocks = 8192;

// Cells per thread of the cell scan: 2, or the smallest power of two that
// keeps the number of scan blocks within kMaxScanBlocks.
inline uint32_t cell_items(uint32_t numCells) {
    uint32_t items = kMinCellItems;
    while ((size_t)numCells > (size_t)kMaxScanBlocks * kThreads * items && items < (1u << 20))
        items <<= 1;
    return items;
}
inline size_t cell_blocks(uint32_t numCells) {
    const size_t chunk = (size_t)kThreads * cell_items(numCells);
    return (numCells + chunk - 1) / chunk;
}
inline unsigned blocks_for(size_t n, int t) { return (unsigned)((n + (size_t)t - 1) / (size_t)t); }
inline uint32_t log2_of(uint32_t pow2) {
    uint32_t k = 0;
    while ((1u << k) < pow2) ++k;
    return k;
}
inline size_t al256(size_t b) { return (b + 255u) & ~(size_t)255u; }

__global__ void fill_u32_kernel(uint32_t* __restrict__ p, uint32_t value, size_t count) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (size_t)gridDim.x * blockDim.x)
        p[i] = value;
}

cudaError_t fill_u32(uint32_t* p, uint32_t value, size_t count, cudaStream_t st, int* launches) {
    if (count == 0) return cudaSuccess;
    const unsigned b = std::min<unsigned>(blocks_for(count, kThreads), 148u * 8u);
    fill_u32_kernel<<<b, kThreads, 0, st>>>(p, value, count);
    if (launches) ++*launches;
    return cudaGetLastError();
}

// Inclusive warp scan of 64-bit values.
__device__ __forceinline__ unsigned long long warp_incl_scan(unsigned long long x) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

template <int THREADS>
__device__ __forceinline__ unsigned long long block_excl_scan64(unsigned long long v,
                                                                unsigned long long* warpTot,
                                                                unsigned long long& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned long long x = warp_incl_scan(v);
    if (lane == 31) warpTot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned long long t = lane < THREADS / 32 ? warpTot[lane] : 0ull;
        t = warp_incl_scan(t);
        if (lane < THREADS / 32) warpTot[lane] = t;
    }
    __syncthreads();
    total = warpTot[THREADS / 32 - 1];
    return (warp > 0 ? warpTot[warp - 1] : 0ull) + x - v;
}

// Sum of one 64-bit value per thread over the block, returned to every
// thread; warpTot is free again when it returns.
template <int THREADS>
__device__ __forceinline__ unsigned long long block_sum64(unsigned long long v,
                                                          unsigned long long* warpTot) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) warpTot[threadIdx.x >> 5] = v;
    __syncthreads();
    unsigned long long t = 0;
#pragma unroll
    for (int w = 0; w < THREADS / 32; ++w) t += warpTot[w];
    __syncthreads();
    return t;
}

// New particle count and arrival count of a cell, packed (count | arrivals << 32).
__device__ __forceinline__ unsigned long long cell_counts(const uint2* __restrict__ prevCells,
                                                          const uint32_t* __restrict__ leavers,
                                                          const uint32_t* __restrict__ arrCnt,
                                                          uint32_t c) {
    const uint2 pr = prevCells[c];
    const uint32_t occ = pr.x < pr.y ? pr.y - pr.x : 0u;
    const uint32_t ac = arrCnt[c];
    const uint32_t cnt = occ - leavers[c] + ac;
    return (unsigned long long)cnt | ((unsigned long long)ac << 32);
}

// Whether no mover left or entered scan tile `tile` (its bit is clear).
__device__ __forceinline__ bool tile_clean(const uint32_t* __restrict__ dirty, uint32_t tile) {
    return dirty != nullptr && ((dirty[tile >> 5] >> (tile & 31u)) & 1u) == 0u;
}

// Every kernel of the incremental path returns at once when the last step
// asked for the full path.  The first one reads that request
// (ctrl[kCtrlNeedFull]), keeps it for the others in ctrl[kCtrlPath] (the full
// path, which may run beside them, clears the request) and passes it to the
// graph's conditional node that runs the full path.
__global__ void __launch_bounds__(kThreads)
cells_reduce_kernel(const uint2* __restrict__ prevCells, const uint32_t* __restrict__ prevFirst,
                    const uint32_t* __restrict__ leavers, const uint32_t* __restrict__ arrCnt,
                    const uint32_t* __restrict__ dirty, uint32_t numCells, uint32_t items,
                    unsigned long long* __restrict__ partials, uint32_t* __restrict__ ctrl,
                    const uint32_t* __restrict__ errFlag, cudaGraphConditionalHandle full,
                    int setFull) {
    // after a sort wait gave up the previous order is not a permutation the
    // incremental path can build on: sort from scratch instead
    const bool needFull = ctrl[kCtrlNeedFull] != 0u ||
                          (errFlag != nullptr && (*errFlag & kSortTimeoutBit) != 0u);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctrl[kCtrlPath] = needFull ? 1u : 0u;
        // the movers' kernels read this copy: place_stayers, which may run
        // beside them, clears the count for the step kernel
        ctrl[kCtrlMoverSnap] = ctrl[kCtrlMovers];
        if (setFull) cudaGraphSetConditional(full, needFull ? 1u : 0u);
    }
    if (needFull) return;
    const size_t base = (size_t)blockIdx.x * kThreads * items;
    if (tile_clean(dirty, blockIdx.x)) {
        // no leavers or arrivals: the tile keeps its particle count
        if (threadIdx.x == 0) {
            const size_t end = min(base + (size_t)kThreads * items, (size_t)numCells);
            partials[blockIdx.x] = (unsigned long long)(prevFirst[end] - prevFirst[base]);
        }
        return;
    }
    __shared__ unsigned long long warpTot[kThreads / 32];
    unsigned long long s = 0;
#pragma unroll 2
    for (uint32_t k = 0; k < items; ++k) {
        const size_t c = base + (size_t)k * kThreads + threadIdx.x;
        if (c < numCells) s += cell_counts(prevCells, leavers, arrCnt, (uint32_t)c);
    }
    const unsigned long long total = block_sum64<kThreads>(s, warpTot);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// New ranges, stayer bases and arrival bases of a tile of kThreads * items
// cells, processed in `items` block-wide slabs so every access is coalesced; the
// per-cell counters are cleared for the next step.
__global__ void __launch_bounds__(kThreads)
cells_apply_kernel(const uint2* __restrict__ prevCells, const uint32_t* __restrict__ prevFirst,
                   uint32_t* __restrict__ leavers, uint32_t* __restrict__ arrCnt,
                   uint32_t* __restrict__ arrLo, uint32_t* __restrict__ dirty,
                   uint32_t numCells, uint32_t items,
                   const unsigned long long* __restrict__ partials,
                   uint2* __restrict__ newCells, uint32_t* __restrict__ newFirst,
                   uint32_t* __restrict__ stayBase, uint2* __restrict__ arrInfo,
                   const uint32_t* __restrict__ ctrl) {
    if (ctrl[kCtrlPath]) return;
    __shared__ unsigned long long warpTot[kThreads / 32];
    const size_t base = (size_t)blockIdx.x * kThreads * items;
    // the tile's first slot and first arrival: the totals of the tiles below
    unsigned long long below = 0;
    for (uint32_t j = threadIdx.x; j < blockIdx.x; j += kThreads) below += partials[j];
    unsigned long long carry = block_sum64<kThreads>(below, warpTot);
    if (tile_clean(dirty, blockIdx.x)) {
        // no leavers or arrivals: every cell keeps its particles, shifted by
        // the movers of the tiles below; no counter to clear
        const uint32_t start0 = (uint32_t)carry, f0 = prevFirst[base];
#pragma unroll 1
        for (uint32_t k = 0; k < items; ++k) {
            const size_t c = base + (size_t)k * kThreads + threadIdx.x;
            if (c >= numCells) break;
            const uint32_t a = prevFirst[c], cnt = prevFirst[c + 1] - a;
            const uint32_t start = start0 + (a - f0);
            newCells[c] = cnt ? make_uint2(start, start + cnt) : make_uint2(kEmptyCell, kEmptyCell);
            newFirst[c] = start;
            if (c == numCells - 1) newFirst[numCells] = start + cnt;
            stayBase[c] = start;
        }
        return;
    }
#pragma unroll 1
    for (uint32_t k = 0; k < items; ++k) {
        const size_t c = base + (size_t)k * kThreads + threadIdx.x;
        const bool valid = c < numCells;
        uint32_t occ = 0, lv = 0, ac = 0, lo = 0;
        if (valid) {
            const uint2 pr = prevCells[c];
            occ = pr.x < pr.y ? pr.y - pr.x : 0u;
            lv = leavers[c];
            ac = arrCnt[c];
            lo = arrLo[c];
        }
        const uint32_t cnt = occ - lv + ac;
        const unsigned long long v = valid ? ((unsigned long long)cnt | ((unsigned long long)ac << 32))
                                           : 0ull;
        unsigned long long total;
        const unsigned long long run = carry + block_excl_scan64<kThreads>(v, warpTot, total);
        if (valid) {
            const uint32_t start = (uint32_t)run, abase = (uint32_t)(run >> 32);
            newCells[c] = cnt ? make_uint2(start, start + cnt) : make_uint2(kEmptyCell, kEmptyCell);
            newFirst[c] = start;
            if (c == numCells - 1) newFirst[numCells] = start + cnt;
            stayBase[c] = (start + lo) | (lv ? kHasLeavers : 0u);
            if (ac) arrInfo[c] = make_uint2(abase, ac);
            if (lv) leavers[c] = 0u;
            if (ac) arrCnt[c] = 0u;
            if (lo) arrLo[c] = 0u;
        }
        carry += total;
        __syncthreads();  // warpTot is reused by the next slab
    }
    // every thread read the tile's bit before the first slab's barrier
    if (dirty && threadIdx.x == 0) atomicAnd(dirty + (blockIdx.x >> 5), ~(1u << (blockIdx.x & 31u)));
}

__global__ void arrivals_scatter_kernel(const uint4* __restrict__ movers,
                                        const uint32_t* __restrict__ ctrl, uint32_t cap,
                                        const uint2* __restrict__ arrInfo,
                                        uint32_t* __restrict__ arrSlots) {
    if (ctrl[kCtrlPath]) return;
    const uint32_t count = min(ctrl[kCtrlMoverSnap], cap);
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < count;
         m += gridDim.x * blockDim.x) {
        const uint4 r = movers[m];
        arrSlots[arrInfo[r.y].x + r.w] = r.x;
    }
}

// A particle's move to its sorted slot: position and radius (what neighbour
// searches read in sorted order) and the slot it came from.
__device__ __forceinline__ void move_particle(uint32_t from, uint32_t dst, const SortMove& m) {
    m.posOut[dst] = m.pos[from];
    m.radiusOut[dst] = m.radius[from];
    m.src[dst] = from;
}

// A mover goes after the arrivals of its new cell with smaller index, and
// after the cell's stayers when it comes from a higher cell.
__global__ void place_movers_kernel(const uint4* __restrict__ movers,
                                    const uint32_t* __restrict__ ctrl, uint32_t cap,
                                    const uint2* __restrict__ arrInfo,
                                    const uint32_t* __restrict__ arrSlots,
                                    const uint2* __restrict__ newCells,
                                    uint32_t* __restrict__ newSortedKey, SortMove mv) {
    if (ctrl[kCtrlPath]) return;
    const uint32_t count = min(ctrl[kCtrlMoverSnap], cap);
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < count;
         m += gridDim.x * blockDim.x) {
        const uint4 r = movers[m];
        const uint2 info = arrInfo[r.y];
        const uint32_t g = min(info.y, kMaxGroup);
        uint32_t rank = 0;
        for (uint32_t k = 0; k < g; ++k) rank += arrSlots[info.x + k] < r.x ? 1u : 0u;
        const uint2 cr = newCells[r.y];
        const uint32_t stay = (cr.y - cr.x) - info.y;
        const uint32_t dst = cr.x + rank + (r.z > r.y ? stay : 0u);
        newSortedKey[dst] = r.y;
        move_particle(r.x, dst, mv);
    }
}

// A stayer keeps its rank among the stayers of its cell.  The particle's
// fields are read together with its keys, before its destination is known,
// so that a thread waits on two rounds of loads instead of three.
__global__ void __launch_bounds__(kThreads)
place_stayers_kernel(uint32_t n, const uint32_t* __restrict__ keys,
                     const uint32_t* __restrict__ prevSortedKey,
                     const uint2* __restrict__ prevCells, const uint32_t* __restrict__ stayBase,
                     uint32_t* __restrict__ newSortedKey, SortMove mv,
                     uint32_t* __restrict__ ctrl) {
    if (ctrl[kCtrlPath]) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) ctrl[kCtrlMovers] = 0u;  // the step kernel counts the next step's movers
    if (i >= n) return;
    const uint32_t o = prevSortedKey[i];
    const uint32_t k = keys[i];
    const float2 p = mv.pos[i];
    const float r = mv.radius[i];
    if (k != o) return;
    const uint32_t os = prevCells[o].x;
    const uint32_t sb = stayBase[o];
    uint32_t rank = i - os;
    if (sb & kHasLeavers) {
        const uint32_t stop = min(i, os + kMaxGroup);
        for (uint32_t j = os; j < stop; ++j) rank -= (keys[j] != prevSortedKey[j]) ? 1u : 0u;
    }
    const uint32_t dst = (sb & ~kHasLeavers) + rank;
    newSortedKey[dst] = o;
    mv.posOut[dst] = p;
    mv.radiusOut[dst] = r;
    mv.src[dst] = i;
}

// First particle of every cell c <= numCells (for an empty cell, that of the
// next non-empty one): the lower bound of c in the sorted keys.
__global__ void cell_first_kernel(const uint32_t* __restrict__ sortedKey, uint32_t n,
                                  uint32_t numCells, uint32_t* __restrict__ first) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c <= numCells;
         c += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = n;
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2;
            if (sortedKey[mid] < c) lo = mid + 1;
            else hi = mid;
        }
        first[c] = lo;
    }
}

// Full path, after the radix sort: cell ranges from the sorted keys, the
// gather by the sorted indices, and the sorted keys kept for the next step.
// Keys and indices are clamped to the cell and particle counts: they always
// are in range unless a wait of the sort gave up (kSortTimeoutBit), when the
// sort's output may hold stale words; the clamps keep every access in bounds
// then (the state is invalid and dem_check says so).
__global__ void __launch_bounds__(kThreads)
full_reorder_kernel(uint32_t n, uint32_t numCells, const uint32_t* __restrict__ hash,
                    const uint32_t* __restrict__ index, uint2* __restrict__ cells,
                    uint32_t* __restrict__ newSortedKey, SortMove mv) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    const uint32_t h = valid ? min(hash[i], numCells - 1u) : 0u;
    uint32_t hp = __shfl_up_sync(0xffffffffu, h, 1);
    if ((threadIdx.x & 31) == 0 && valid && i > 0) hp = min(hash[i - 1], numCells - 1u);
    if (!valid) return;
    if (i == 0 || h != hp) {
        cells[h].x = i;
        if (i > 0) cells[hp].y = i;
    }
    if (i == n - 1) cells[h].y = i + 1;
    newSortedKey[i] = h;
    move_particle(min(index[i], n - 1u), i, mv);
}

}  // namespace

size_t incsort_bytes(uint32_t n, uint32_t numCells, uint32_t* moverCapOut) {
    const uint32_t cap = std::max<uint32_t>(4096u, n / 8u);
    if (moverCapOut) *moverCapOut = cap;
    const size_t cells = al256(4ull * numCells);
    const size_t np = cell_blocks(numCells);
    return 4 * cells + al256(8ull * numCells) + al256(16ull * cap) + al256(4ull * cap) +
           al256(8ull * std::max<size_t>(np, 1)) + al256(4ull * ((np + 31) / 32 + 1)) + 256;
}

IncSort carve_incsort(void* base, uint32_t n, uint32_t numCells) {
    IncSort s;
    s.numCells = numCells;
    incsort_bytes(n, numCells, &s.moverCap);
    const size_t cells = al256(4ull * numCells);
    const size_t np = cell_blocks(numCells);
    char* p = static_cast<char*>(base);
    s.leavers = reinterpret_cast<uint32_t*>(p); p += cells;
    s.arrCnt = reinterpret_cast<uint32_t*>(p); p += cells;
    s.arrLo = reinterpret_cast<uint32_t*>(p); p += cells;
    s.stayBase = reinterpret_cast<uint32_t*>(p); p += cells;
    s.arrInfo = reinterpret_cast<uint2*>(p); p += al256(8ull * numCells);
    s.movers = reinterpret_cast<uint4*>(p); p += al256(16ull * s.moverCap);
    s.arrSlots = reinterpret_cast<uint32_t*>(p); p += al256(4ull * s.moverCap);
    s.partials = reinterpret_cast<unsigned long long*>(p); p += al256(8ull * std::max<size_t>(np, 1));
    s.dirty = reinterpret_cast<uint32_t*>(p); p += al256(4ull * ((np + 31) / 32 + 1));
    s.tileShift = log2_of(kThreads * cell_items(numCells));
    s.ctrl = reinterpret_cast<uint32_t*>(p);
    return s;
}

cudaError_t enqueue_incremental_head(const IncSort& s, const uint2* prevCells,
                                     const uint32_t* prevFirst, cudaGraphConditionalHandle full,
                                     bool setFull, cudaStream_t st, int* launches) {
    const uint32_t C = s.numCells;
    const size_t nb = cell_blocks(C);
    if (nb > kMaxScanBlocks) return cudaErrorInvalidValue;
    cells_reduce_kernel<<<(unsigned)nb, kThreads, 0, st>>>(prevCells, prevFirst, s.leavers,
                                                           s.arrCnt, s.dirty, C, cell_items(C),
                                                           s.partials, s.ctrl, s.errFlag, full,
                                                           setFull ? 1 : 0);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t enqueue_incremental_tail(const IncSort& s, uint32_t n, const uint32_t* keys,
                                     const uint32_t* prevSortedKey, const uint2* prevCells,
                                     const uint32_t* prevFirst, uint32_t* newSortedKey, uint2* newCells, uint32_t* newFirst,
                                     const SortMove& mv, cudaStream_t st, int* launches,
                                     cudaStream_t side, cudaEvent_t forkEv, cudaEvent_t joinEv) {
    const uint32_t C = s.numCells;
    const uint32_t items = cell_items(C);
    const size_t nb = cell_blocks(C);
    if (nb > kMaxScanBlocks) return cudaErrorInvalidValue;
    cells_apply_kernel<<<(unsigned)nb, kThreads, 0, st>>>(prevCells, prevFirst, s.leavers,
                                                          s.arrCnt, s.arrLo, s.dirty, C, items,
                                                          s.partials, newCells, newFirst,
                                                          s.stayBase, s.arrInfo, s.ctrl);
    // the movers (two small kernels) on `side` when given, beside the
    // stayers: both only read what cells_apply wrote, and write disjoint slots
    const bool fork = side && forkEv && joinEv;
    cudaStream_t ms = st;
    if (fork) {
        cudaError_t e = cudaEventRecord(forkEv, st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(side, forkEv, 0);
        if (e != cudaSuccess) return e;
        ms = side;
    }
    const unsigned mb = std::min<unsigned>(blocks_for(s.moverCap, kThreads), 296u);
    arrivals_scatter_kernel<<<mb, kThreads, 0, ms>>>(s.movers, s.ctrl, s.moverCap, s.arrInfo,
                                                     s.arrSlots);
    place_movers_kernel<<<mb, kThreads, 0, ms>>>(s.movers, s.ctrl, s.moverCap, s.arrInfo,
                                                 s.arrSlots, newCells, newSortedKey, mv);
    if (n) {
        place_stayers_kernel<<<blocks_for(n, kThreads), kThreads, 0, st>>>(
            n, keys, prevSortedKey, prevCells, s.stayBase, newSortedKey, mv, s.ctrl);
    }
    if (launches) *launches += 4;
    cudaError_t e = cudaGetLastError();
    if (fork) {
        // join the movers' branch even after an error
        cudaError_t ej = cudaEventRecord(joinEv, side);
        if (ej == cudaSuccess) ej = cudaStreamWaitEvent(st, joinEv, 0);
        if (e == cudaSuccess) e = ej;
    }
    return e;
}

cudaError_t enqueue_full(const IncSort& s, uint32_t n, uint32_t keyBits, uint32_t* keys,
                         uint32_t* perm, const OnesweepScratch& os, uint32_t* errFlag,
                         uint32_t* newSortedKey, uint2* newCells, uint32_t* newFirst,
                         const SortMove& mv, cudaStream_t st, int* launches) {
    uint32_t *ko, *vo;
    cudaError_t e = onesweep_sort_pairs(keys, perm, n, keyBits, true, os, errFlag, st, &ko, &vo,
                                        launches);
    if (e != cudaSuccess) return e;
    e = fill_u32(reinterpret_cast<uint32_t*>(newCells), kEmptyCell, 2ull * s.numCells, st,
                 launches);
    if (e != cudaSuccess) return e;
    if (n) {
        full_reorder_kernel<<<blocks_for(n, kThreads), kThreads, 0, st>>>(
            n, s.numCells, ko, vo, newCells, newSortedKey, mv);
        if (launches) ++*launches;
    }
    cell_first_kernel<<<std::min<unsigned>(blocks_for((size_t)s.numCells + 1, kThreads), 148u * 8u),
                        kThreads, 0, st>>>(newSortedKey, n, s.numCells, newFirst);
    if (launches) ++*launches;
    // the incremental counters restart from zero: the step kernel of this
    // step records the movers of the next one
    e = fill_u32(s.leavers, 0u, s.numCells, st, launches);
    if (e == cudaSuccess) e = fill_u32(s.arrCnt, 0u, s.numCells, st, launches);
    if (e == cudaSuccess) e = fill_u32(s.arrLo, 0u, s.numCells, st, launches);
    if (e == cudaSuccess) e = fill_u32(s.ctrl, 0u, 2, st, launches);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace dem
