// Kernel launchers for the DEM step (definitions in dem_kernels.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dem_common.cuh"

namespace dem {

// Pointers of one state set in the reference SoA layout.
struct DynSet {
    float2* pos;
    float2* vel;
    float* theta;
    float* omega;
};
struct StatSet {
    float* radius;
    float* mass;
    uint32_t* id;
    uint32_t* type;  // may be null (single material)
};

constexpr uint32_t kFollowBatch = 64;
struct FollowIds {
    uint32_t count;
    uint32_t id[kFollowBatch];
};
cudaError_t launch_followed(const FollowIds& f, const uint32_t* loc, DynSet d, StatSet s,
                            const float2* acc, const float* alpha, const float* pressure,
                            float* rows, cudaStream_t st);
// Followed rows of a multi-step call: the ids ids[0, *countWord) (device
// memory) gathered into row block (slot ? *slot : 0) + add of `ring`, each
// block *countWord rows of 12 words (the device-side loop advances *slot).
cudaError_t launch_followed_ring(const uint32_t* ids, const uint32_t* countWord,
                                 const uint32_t* slot, uint32_t add, const uint32_t* loc, DynSet d,
                                 StatSet s, const float2* acc, const float* alpha,
                                 const float* pressure, float* ring, cudaStream_t st);

// Upper bound of the radii: writes the largest radius's bit pattern to *out.
cudaError_t launch_max_radius(const float* radius, uint32_t n, uint32_t* out, cudaStream_t st);

cudaError_t launch_calc_hash(const KParams& P, const float2* pos, uint32_t* hash, uint32_t* index,
                             uint32_t n, cudaStream_t st);
cudaError_t launch_calc_hash_batched(const KParams* table, const uint32_t* spec, const float2* pos,
                                     uint32_t* hash, uint32_t n, cudaStream_t st);

cudaError_t launch_reorder(const KParams& P, uint32_t* cellStart, uint32_t* cellEnd,
                           DynSet sorted, StatSet sortedS, uint32_t* sortedLoc,
                           const uint32_t* hash, const uint32_t* index, DynSet old, StatSet oldS,
                           uint32_t n, uint32_t numCells, bool clearCells, cudaStream_t st,
                           int* launches);

cudaError_t launch_collide(const KParams& P, const float2* pos, const float2* vel,
                           const float* omega, const float* radius, const float* mass,
                           const uint32_t* type, const uint32_t* cellStart,
                           const uint32_t* cellEnd, float2* acc, float* alpha, float* pressure,
                           uint32_t n, cudaStream_t st);

cudaError_t launch_integrate(const KParams& P, float2* pos, float2* vel, const float2* acc,
                             float* theta, float* omega, const float* alpha, const uint32_t* type,
                             const float* radius, const float* mass, float* pressure, uint32_t n,
                             cudaStream_t st);

// Fused collide + integrate + next-step hash: reads the sorted set `in`
// (with its sort keys and interleaved cell ranges), writes the integrated
// state to `out` (same order) and the cell key of each new position to
// `nextHash`.  acc/alpha/pressure may be null.
// Movers (particles whose cell changes) are reported to `sink` for the
// incremental sort; a null sink.ctrl disables the recording.
struct MoverSinkArgs {
    uint32_t* leavers;
    uint32_t* arrCnt;
    uint32_t* arrLo;
    uint4* movers;
    uint32_t* ctrl;
    uint32_t moverCap;
    uint32_t tileShift;  // cells per tile of the cell scan: 2^tileShift
    uint32_t* dirty;     // a bit per tile holding a mover's old or new cell (may be null)
};
// The control ("big") particle of the reference built with USE_BIG_PARTICLE 1
// (device memory, read by the step kernel and moved by control_move_kernel).
struct ControlDev {
    float2 pos, vel;
    float theta, omega, radius;
    uint32_t mat;
    double drift[2];
    double wrapYBelow, wrapYTo, wrapXAbove, wrapXTo;  // NaN: no wrap
};
// Step-kernel outputs of the control particle: per-particle reaction
// vectors (-f.x, -f.y, -m / r * rControl), or c == null when there is none.
struct ControlArgs {
    const ControlDev* c;
    float* fx;
    float* fy;
    float* fm;
};
// The context step kernel.  in.pos and inS.radius are in this step's sorted
// order; the particle at sorted slot i has its other fields (in.vel, theta,
// omega, inS.mass, id, type) at slot src[i] of the previous order.  The new
// state is written in the sorted order: positions, velocities, angles and
// spins to `out`, mass, id and type to `outS`, and loc[id] = slot.
// cellRange: (start, end) of every cell; cellFirst: numCells + 4 words, the
// first particle of every cell (for an empty cell, that of the next
// non-empty one) and n at [numCells].
cudaError_t launch_step(const KParams& P, DynSet in, StatSet inS, const uint32_t* src,
                        const uint32_t* sortedKey, const uint2* cellRange,
                        const uint32_t* cellFirst, DynSet out, StatSet outS, uint32_t* loc,
                        uint32_t* nextHash, float* pressure, float2* acc, float* alpha,
                        uint32_t* errFlag, uint32_t n, MoverSinkArgs sink, cudaStream_t st,
                        const KParams* table = nullptr, const uint32_t* spec = nullptr,
                        ControlArgs ctl = ControlArgs{}, int variant = 0);
// Launch shapes of the step kernel: threads per block x the blocks per SM its
// registers are capped for (variant 0: 128 x 8, 1: 64 x 16, 2: 256 x 4,
// 3: 128 x 6, which allows 80 registers).  All compute the same bits; the
// control-particle step always runs variant 0's shape.
constexpr int kStepVariants = 4;
// Elements of padding after the sorted positions and radii of a context:
// the step kernel's candidate filter reads whole groups of 8 candidates.
constexpr uint32_t kFilterPad = 8;
struct StepShape {
    int threads, blocksPerSm;
};
StepShape step_variant_shape(int variant);
// After the step kernel: the reaction sums (reduceVecD's blocks, then their
// sum in block order: out[0..2] = force x, force y, moment) and the control
// particle's move.  partials: 3 * ceil(n / min(512, n)) floats.
cudaError_t launch_control_post(ControlArgs ctl, ControlDev* c, uint32_t n, float* partials,
                                float* out, cudaStream_t st, int* launches);

// Reorder with interleaved (start, end) cell ranges; resets the ranges first.
cudaError_t launch_reorder_packed(uint2* cellRange, DynSet sorted, StatSet sortedS,
                                  uint32_t* sortedLoc, const uint32_t* hash, const uint32_t* index,
                                  DynSet old, StatSet oldS, uint32_t n, uint32_t numCells,
                                  cudaStream_t st, int* launches);

// Splits interleaved ranges into the reference's cellStart/cellEnd arrays.
cudaError_t launch_unpack_cells(const uint2* cellRange, uint32_t numCells, uint32_t* cellStart,
                                uint32_t* cellEnd, cudaStream_t st);

// Device-side loops (a WHILE node of a graph): loop_init copies the
// requested count of iterations (*req) to *left and sets the node's
// condition; loop_next, the last kernel of each iteration, counts one down,
// adds idxStep to *idx (when idx is not null: the loop's record slot) and
// sets the condition again.
cudaError_t launch_loop_init(const uint32_t* req, uint32_t* left, cudaGraphConditionalHandle h,
                             cudaStream_t st);
cudaError_t launch_loop_next(uint32_t* left, uint32_t* idx, int32_t idxStep,
                             cudaGraphConditionalHandle h, cudaStream_t st);
// Writes up to 8 words, passed by value, to device memory in stream order
// (a loop's counts before its launch: no host buffer has to outlive the
// call, and the host never waits).
struct Words {
    uint32_t v[8];
    uint32_t count;
};
cudaError_t launch_set_words(uint32_t* dst, Words w, cudaStream_t st);

// Adjoint (dem_adjoint.cu).
size_t adj_step_bytes(uint32_t n, uint32_t numCells);
// Writes the record of one forward step at recBase in one launch: the sorted
// state the step kernel stepped (d, s and src as launch_step's in, inS and
// src), its cell ranges and the acceleration and angular acceleration it
// produced.
// The record a kernel reads or writes: recBase itself, or, with `slot`
// set, the record of step (*slot + add) of a window whose records are
// `stride` bytes apart from recBase -- the form a device-side loop uses,
// its slot advanced by loop_next.
struct RecSlot {
    const uint32_t* slot = nullptr;
    uint32_t add = 0;
    size_t stride = 0;
};
cudaError_t adj_record_step(void* recBase, RecSlot at, uint32_t n, uint32_t numCells, DynSet d,
                            StatSet s, const uint32_t* src, const uint2* cells, const float2* acc,
                            const float* alpha, cudaStream_t st);
// table/spec: the batch's specimen table and slot -> specimen map, or null
// for a single scene (then P).
cudaError_t adj_backward_step(const KParams& P, const KParams* table, const uint32_t* spec,
                              void* recBase, RecSlot at, uint32_t n, uint32_t numCells,
                              float2* lamX, float2* lamV, float* lamW, float2* tlx, float2* tlv,
                              float* tlw, float2* lamF, float* lamM, double* acc, cudaStream_t st);
// Per-specimen coefficient gradients (first: numSpecimens + 1 slot offsets,
// or null for one specimen of n slots).
cudaError_t adj_sum_coef(const double* acc, uint32_t n, const uint32_t* first, uint32_t numSpecimens,
                         double* out, cudaStream_t st);
size_t adj_acc_bytes(uint32_t n);

// Disk splat of n particles into a DIMx x DIMy uchar4 image (dem_render.cu);
// owner: DIMx * DIMy words of scratch.
cudaError_t launch_render(const DemRenderParams& rp, float Lx, float Ly, const float2* pos,
                          const float* theta, const uint32_t* type, const float* radius,
                          const float* pressure, uint32_t n, uint32_t* owner, uchar4* image,
                          cudaStream_t st);

}  // namespace dem
