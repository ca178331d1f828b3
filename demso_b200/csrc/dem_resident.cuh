// Resident batched step: a multi-step call of a batch run as one persistent
// launch in which every specimen lives in one streaming multiprocessor's
// shared memory for all of its steps (definitions in dem_resident.cu).
#pragma once

#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "dem_kernels.cuh"

namespace dem {

// Limits of one bin (the specimens a thread block steps together in shared
// memory): particles, cells and specimens.  24 B per particle (position,
// velocity, spin, radius) and 4 B per cell (first-particle array) fit the
// 227 KB of shared memory a block of an sm_100 multiprocessor may hold.
constexpr uint32_t kResMaxParticles = 8192;
constexpr uint32_t kResMaxCells = 8192;
constexpr uint32_t kResMaxEntries = 64;

// One specimen of a bin: its index in the batch, its first slot in the
// batch's state and in the bin, its particle count, and its first cell in the
// bin's cell numbering and cell count.
struct ResEntry {
    uint32_t spec, gslot, slot, n, cellOff, cells;
};
// A bin: entries [first, first + count) of the entry array, its particles and
// cells.
struct ResBin {
    uint32_t first, count, n, cells;
};

// The batch's current state (order of the last sort) that the launch reads at
// the start and writes back at the end, and the outputs of its last step.
struct ResIO {
    float2* pos;
    float2* vel;
    float* theta;
    float* omega;
    float* radius;
    float* mass;
    uint32_t* id;
    uint32_t* loc;
    float* pressure;  // may be null
    float2* acc;      // may be null
    float* alpha;     // may be null
};

// Packs specimens (first slots partOff[0..nspec], cells per specimen) into
// bins, largest specimen first into the first bin with room, and orders the
// bins by particle count, largest first.  Returns false when a specimen does
// not fit one bin.
bool resident_plan(const std::vector<uint32_t>& partOff, const std::vector<uint32_t>& cells,
                   std::vector<ResEntry>& entries, std::vector<ResBin>& bins, uint32_t& maxN,
                   uint32_t& maxC);

// Per-block global scratch of a launch whose largest bin holds maxN particles.
size_t resident_work_bytes(uint32_t maxN);
// Shared memory of one block for bins of up to maxN particles and maxC cells.
size_t resident_smem_bytes(uint32_t maxN, uint32_t maxC);
// Blocks of a launch on this device (one per multiprocessor, at most the bins).
int resident_blocks(uint32_t numBins, int device);

// `nsteps` steps of every bin; `queue` is one device word (zeroed here, on
// `st`), `work` resident_work_bytes(maxN) bytes per block; nTotal is the
// batch's particle count (ids index loc below it).
cudaError_t launch_resident(const KParams* table, const ResBin* bins, uint32_t numBins,
                            const ResEntry* entries, uint32_t maxN, uint32_t maxC,
                            uint32_t* queue, void* work, int blocks, ResIO io, uint32_t nTotal,
                            uint32_t nsteps, uint32_t* errFlag, cudaStream_t st);


// One scene stepped by a thread-block cluster (every block a full copy of
// the scene in its shared memory, its own share of the slots stepped, the
// new state broadcast through distributed shared memory).  Fits scenes of at
// most kResMaxParticles disks and kResMaxCells cells; `work` is
// cluster_scene_work_bytes(n) bytes of device memory.  Returns
// cudaErrorNotSupported when no cluster of this shape can be resident.
bool cluster_scene_fits(uint32_t n, uint32_t cells);
size_t cluster_scene_work_bytes(uint32_t n);
cudaError_t launch_cluster_scene(const KParams& P, uint32_t n, uint32_t cells, void* work,
                                 ResIO io, uint32_t nsteps, uint32_t* errFlag, cudaStream_t st);

}  // namespace dem
