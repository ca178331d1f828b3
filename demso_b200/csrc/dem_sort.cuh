// In-house stable LSD radix sort of (uint32 key, uint32 value) pairs.
//
// Replaces thrust::sort_by_key in the reference (functions.cu:336-341), which
// is a stable ascending radix sort.  Each pass is reduce-then-scan:
//   upsweep   : per-tile digit histogram, stored digit-major [digit][tile]
//   scan      : one exclusive scan over that table (global digit offsets)
//   downsweep : per-tile stable ranking with warp match_any, then scatter
// so there are no inter-block waits at all.  Digit width adapts to the key
// width: ceil(keyBits / 11) passes of at most 11 bits each (the 20-bit cell
// keys of a 1024x1024 grid take two 10-bit passes).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace dem {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys per tile
constexpr int kSortWarps = kSortThreads / 32;

struct SortPlan {
    int passes = 0;
    int shift[4] = {0, 0, 0, 0};
    int bits[4] = {0, 0, 0, 0};
    int radixBits = 0;  // template width used for every pass (>= bits[p])
};

SortPlan make_sort_plan(uint32_t keyBits);
size_t sort_hist_words(uint32_t n, const SortPlan& plan);
size_t sort_scan_partials(size_t words);

struct SortScratch {
    uint32_t* altKeys;   // n
    uint32_t* altVals;   // n
    uint32_t* hist;      // sort_hist_words
    uint32_t* partials;  // sort_scan_partials
};

// Bytes of scratch for the layout carve_sort_scratch produces.
size_t sort_scratch_bytes(uint32_t n, uint32_t keyBits);
SortScratch carve_sort_scratch(void* base, uint32_t n, uint32_t keyBits);

// Sorts keys/vals of length n.  When `identityVals` is true the input values
// are not read: value i is taken to be i (what calcHash writes).  On return
// the sorted pairs are in (*keysOut, *valsOut), which point either at the
// inputs or at the scratch alternates, depending on the pass count.
cudaError_t radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t keyBits,
                             bool identityVals, const SortScratch& s, cudaStream_t stream,
                             uint32_t** keysOut, uint32_t** valsOut, int* launches);

// Single-pass-per-digit variant ("onesweep"): one kernel computes the global
// digit histograms of every pass from the input keys, then each pass is one
// kernel whose tiles take their digit offsets from their predecessors by
// decoupled look-back.  Tiles are numbered in launch order by an atomic
// counter, so a tile only ever waits on tiles that are already running;
// every wait is bounded and, if it gives up, sets kSortTimeoutBit in
// *errFlag and carries on (the result is then invalid, never a hang).
constexpr uint32_t kSortTimeoutBit = 2u;
// Iterations a look-back wait spins (with short sleeps) before it gives up.
constexpr uint32_t kSortSpinLimit = 1u << 22;
constexpr uint32_t kNoHeldTile = 0xffffffffu;

struct OnesweepScratch {
    uint32_t* altKeys;    // n
    uint32_t* altVals;    // n
    uint32_t* globalHist; // passes * 2^maxBits (exclusive offsets after the scan)
    uint32_t* lookback;   // 1 counter word padded to 64, then numTiles * 2^maxBits
    // Test hook (dem_debug_sort_hold): tile `holdTile` of every pass never
    // publishes its counts, so the tile after it waits until `spinLimit`
    // runs out; kNoHeldTile and kSortSpinLimit in normal use.
    uint32_t holdTile = kNoHeldTile;
    uint32_t spinLimit = kSortSpinLimit;
};
size_t onesweep_scratch_bytes(uint32_t n, uint32_t keyBits);
OnesweepScratch carve_onesweep_scratch(void* base, uint32_t n, uint32_t keyBits);
cudaError_t onesweep_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t keyBits,
                                bool identityVals, const OnesweepScratch& s, uint32_t* errFlag,
                                cudaStream_t stream, uint32_t** keysOut, uint32_t** valsOut,
                                int* launches);

// Exclusive scan of `len` words in place; partials holds sort_scan_partials(len).
cudaError_t exclusive_scan_u32(uint32_t* data, size_t len, uint32_t* partials,
                               cudaStream_t stream, int* launches);

}  // namespace dem
