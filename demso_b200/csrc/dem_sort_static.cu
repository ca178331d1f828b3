// dem_sort_particles_static: the stable radix sort of dem_sort_particles for
// callers that cannot allocate device memory.
//
// Some callers of a sort like this cannot call cudaMalloc or take scratch
// from an allocator: step loops that must not stall on the device-wide
// synchronisation cudaMalloc/cudaFree can imply, and host programs whose own
// memory manager owns every device allocation and hands out no scratch.  This
// variant takes its scratch from a fixed array in the library's device
// memory instead.  Only the caller's inputs/outputs are passed in.
//
// The array is sized for kStaticSortMaxPairs pairs of any key width (about
// 2.6 MB).  Every GPU that loads the library holds it until the process
// exits.  All calls share it, so calls whose execution overlaps on the GPU
// (other streams, other host threads, same device) race on it and corrupt
// each other's results; order them on one stream or synchronise between
// them.  Every scratch word is written before it is read within a call (the
// per-tile histograms, the scan partials and the alternate key/value
// buffers), so nothing left from an earlier call needs clearing.
#include <cstdio>
#include <mutex>

#include "../../include/demso_b200.h"
#include "dem_sort.cuh"

// Records the message returned by dem_last_error_string (dem_api.cu).
int dem_record_error(int code, const char* msg);

namespace {

constexpr uint32_t kStaticSortMaxPairs = 1u << 18;
constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t b) { return (b + kAlign - 1) & ~(kAlign - 1); }
// The layout carve_sort_scratch produces at the largest size: two alternate
// arrays of n words, the per-tile digit histograms (at most 11-bit digits)
// and the scan partials.
constexpr size_t kTiles = (kStaticSortMaxPairs + dem::kSortTile - 1) / dem::kSortTile;
constexpr size_t kHistWords = kTiles * 2048;
constexpr size_t kPartials = (kHistWords + 4095) / 4096;
constexpr size_t kStaticSortScratchBytes = 2 * align_up(4 * (size_t)kStaticSortMaxPairs) +
                                           align_up(4 * kHistWords) + align_up(4 * kPartials);

static __device__ __align__(256) unsigned char g_sortScratch[kStaticSortScratchBytes];

// Device address of g_sortScratch, looked up once per device.  In host code
// the symbol names a host-side stand-in, not device memory, so the kernels
// must be given this address instead.  It is kept for the life of the
// process, so a device reset after the first call (which would free the
// module's memory and load it again elsewhere) is not supported.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratchPtr[kMaxDevices] = {};

cudaError_t scratch_for_current_device(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratchPtr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sortScratch);
        if (e != cudaSuccess) return e;
        g_scratchPtr[dev] = p;
    }
    *out = g_scratchPtr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" int dem_sort_particles_static(uint32_t* gridParticleHash, uint32_t* gridParticleIndex,
                                         uint32_t numParticles, uint32_t keyBits, void* stream) {
    char msg[256];
    if (keyBits > 32) {
        snprintf(msg, sizeof(msg), "keyBits %u > 32", keyBits);
        return dem_record_error(DEM_ERR_INVALID_ARG, msg);
    }
    if (numParticles > kStaticSortMaxPairs) {
        snprintf(msg, sizeof(msg),
                 "dem_sort_particles_static: %u pairs exceed the fixed scratch (at most %u); "
                 "use dem_sort_particles with caller scratch",
                 numParticles, kStaticSortMaxPairs);
        return dem_record_error(DEM_ERR_CAPACITY, msg);
    }
    if (numParticles == 0) return DEM_OK;
    if (!gridParticleHash || !gridParticleIndex)
        return dem_record_error(DEM_ERR_INVALID_ARG, "dem_sort_particles_static: NULL buffer");
    if (dem::sort_scratch_bytes(numParticles, keyBits) > kStaticSortScratchBytes)
        return dem_record_error(DEM_ERR_CAPACITY,
                                "dem_sort_particles_static: scratch layout too large");
    void* base = nullptr;
    cudaError_t e = scratch_for_current_device(&base);
    if (e != cudaSuccess) {
        snprintf(msg, sizeof(msg), "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        return dem_record_error(DEM_ERR_CUDA, msg);
    }
    const dem::SortScratch s = dem::carve_sort_scratch(base, numParticles, keyBits);
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t *ko, *vo;
    e = dem::radix_sort_pairs(gridParticleHash, gridParticleIndex, numParticles, keyBits, false, s,
                              st, &ko, &vo, nullptr);
    if (e == cudaSuccess && ko != gridParticleHash) {
        e = cudaMemcpyAsync(gridParticleHash, ko, sizeof(uint32_t) * numParticles,
                            cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(gridParticleIndex, vo, sizeof(uint32_t) * numParticles,
                                cudaMemcpyDeviceToDevice, st);
    }
    if (e != cudaSuccess) {
        snprintf(msg, sizeof(msg), "radix sort: %s", cudaGetErrorString(e));
        return dem_record_error(DEM_ERR_CUDA, msg);
    }
    return DEM_OK;
}
