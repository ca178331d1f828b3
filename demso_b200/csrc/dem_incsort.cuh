// Incremental stable sort of the context step.
//
// Between two steps a particle changes cell only when it crosses a cell
// border, which in a granular packing is rare.  The state is kept sorted by
// cell, and the stable sort of the new keys is rebuilt from the old order:
// for each cell c the stable order is
//     [arrivals from cells < c, by index] [stayers of c, in old order]
//     [arrivals from cells > c, by index]
// because the old order is sorted by old cell.  The step kernel records every
// particle whose cell changes ("mover") with its old and new cell and a slot
// in the new cell's arrival group, and counts leavers/arrivals per cell.
// Then:
//   cells pass  : new count per cell = old count - leavers + arrivals, and
//                 an exclusive scan of (count, arrivals) gives each cell's
//                 start and its arrivals' base;
//   movers      : each mover's rank among its cell's arrivals by index;
//   placement   : every particle computes its sorted position and moves its
//                 position and radius there (scatter, nearly coalesced),
//                 with its sorted key and the slot it came from; the step
//                 kernel gathers the other fields through that slot.
// The result is identical to the stable radix sort + reorder of the
// reference.  When the mover list overflows, an arrival group or a leaving
// cell is larger than kMaxGroup, or there is no previous order (first
// step), the full path runs instead: the onesweep radix sort, cell ranges
// from the sorted keys, and the gather.  The incremental kernels run
// unconditionally and return at once when the full path is due; the full
// path sits in a graph conditional node that the first of them switches on.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dem_kernels.cuh"
#include "dem_sort.cuh"

namespace dem {

constexpr uint32_t kCtrlNeedFull = 0;        // ctrl[0]: non-zero -> full path next step
constexpr uint32_t kCtrlMovers = 1;          // ctrl[1]: movers recorded by the step kernel
constexpr uint32_t kCtrlPath = 2;            // ctrl[2]: this step runs the full path
constexpr uint32_t kCtrlMoverSnap = 3;       // ctrl[3]: this step's movers, kept by the first kernel
constexpr uint32_t kHasLeavers = 0x80000000u;  // flag bit in stayBase

// The state the sort phase moves: positions and radii from the previous
// order to the sorted one, and for every sorted slot the previous slot of
// its particle (src).
struct SortMove {
    const float2* pos;
    const float* radius;
    float2* posOut;
    float* radiusOut;
    uint32_t* src;
};

// Buffers of the incremental path (all device memory, owned by the context).
struct IncSort {
    uint32_t numCells = 0, moverCap = 0;
    uint32_t* leavers = nullptr;   // per cell, zero between steps
    uint32_t* arrCnt = nullptr;    // per cell, zero between steps
    uint32_t* arrLo = nullptr;     // per cell, zero between steps
    uint32_t* stayBase = nullptr;  // per cell
    uint2* arrInfo = nullptr;      // per cell (written for cells with arrivals)
    uint4* movers = nullptr;       // moverCap records (index, new cell, old cell, arrival slot)
    uint32_t* arrSlots = nullptr;  // moverCap
    unsigned long long* partials = nullptr;  // scan partials
    // A bit per scan tile (the 2^tileShift cells a block of the cell scan
    // takes) set by the step kernel for the old and the new cell of every
    // mover; the cell scan takes a clean tile's ranges from the previous
    // first-particle array, shifted, and clears the bits of the tiles it
    // scanned.  A stale bit only sends a tile through the full scan.
    uint32_t* dirty = nullptr;
    uint32_t tileShift = 0;
    uint32_t* ctrl = nullptr;      // kCtrlNeedFull, kCtrlMovers, kCtrlPath
    // the context's error word: while a sort wait has given up
    // (kSortTimeoutBit), every step takes the full path, which needs no
    // previous order (set by the context after carve_incsort)
    const uint32_t* errFlag = nullptr;
};

size_t incsort_bytes(uint32_t n, uint32_t numCells, uint32_t* moverCapOut);
IncSort carve_incsort(void* base, uint32_t n, uint32_t numCells);

// Fast path: new cell ranges, sorted keys, moved state.  prev* describe the
// order the step kernel just stepped (prevFirst: its first-particle array,
// numCells + 1 entries); `keys` are the new keys.  `head` (the
// first kernel) reads whether the full path is due, keeps the answer in
// ctrl[kCtrlPath] for the kernels of `tail`, and with setFull passes it to
// the graph conditional handle `full`.  With a `side` stream (and two events)
// `tail` places the movers on it, beside the stayers on `st` -- the two write
// disjoint slots -- and joins it back into `st` before returning.
cudaError_t enqueue_incremental_head(const IncSort& s, const uint2* prevCells,
                                     const uint32_t* prevFirst, cudaGraphConditionalHandle full,
                                     bool setFull, cudaStream_t st, int* launches);
cudaError_t enqueue_incremental_tail(const IncSort& s, uint32_t n, const uint32_t* keys,
                                     const uint32_t* prevSortedKey, const uint2* prevCells,
                                     const uint32_t* prevFirst,
                                     uint32_t* newSortedKey, uint2* newCells, uint32_t* newFirst,
                                     const SortMove& mv, cudaStream_t st, int* launches,
                                     cudaStream_t side = nullptr, cudaEvent_t forkEv = nullptr,
                                     cudaEvent_t joinEv = nullptr);

// Full path: onesweep sort of `keys`, cell ranges, gather, reset of the
// incremental counters.  `perm` and `keys` are overwritten.
cudaError_t enqueue_full(const IncSort& s, uint32_t n, uint32_t keyBits, uint32_t* keys,
                         uint32_t* perm, const OnesweepScratch& os, uint32_t* errFlag,
                         uint32_t* newSortedKey, uint2* newCells, uint32_t* newFirst,
                         const SortMove& mv, cudaStream_t st, int* launches);

}  // namespace dem
