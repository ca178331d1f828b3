// Resident batched step (DEM_CTX_RESIDENT): a multi-step dem_step call of a
// batch runs as ONE persistent launch.  Specimens are packed into bins of up
// to kResMaxParticles particles and kResMaxCells cells; each thread block
// (one per multiprocessor, 1024 threads) takes bins from a queue, loads a
// bin's state into shared memory and runs every step of the call there:
//
//   sort     : only when some particle changed cell in the last step (and
//              on the first step): a stable block-wide sort of the slots by
//              cell -- one-bit LSD passes over the cell bits that differ,
//              with warp ballots -- then the first-particle array of every
//              cell and the state gathered into the new order;
//   collide  : every particle against the particles of its 3 x 3 cells,
//              cells y-outer, x-inner, each cell's particles in slot order,
//              one subtotal per cell (collideD, particles_kernel.cuh:459-549,
//              with collideCell :346-385 and collideSpheres :236-307), the
//              neighbours read from shared memory; forces, moments and
//              pressures to the block's scratch;
//   integrate: integrateSystemD + collideBoundary (particles_kernel.cuh:
//              388-456, 580-627) in place, then the particle's new cell.
//
// The sort is the reference's stable sort by cell restricted to the bin, and
// the sums are added in the reference's order, so every specimen follows the
// same trajectory bit for bit as in the graph path of the batch or alone.
// Velocities, spins, radii and positions -- what neighbours read -- live in
// shared memory (24 B per particle); angles, masses and ids are read and
// written only by the particle's own thread and live in the block's global
// scratch, which stays in L2.
//
// The same file steps a single scene of up to kResMaxParticles disks as one
// thread-block cluster (cluster_kernel, below): every block holds the whole
// scene, steps its share of the slots and broadcasts their new state to the
// other blocks through distributed shared memory.
#include <algorithm>

#include <cooperative_groups.h>

#include "dem_resident.cuh"

namespace cg = cooperative_groups;

namespace dem {
namespace {

#ifndef DEM_RES_THREADS
#define DEM_RES_THREADS 1024
#endif
constexpr int kResThreads = DEM_RES_THREADS;  // one block per multiprocessor
constexpr int kResWarps = kResThreads / 32;
constexpr uint32_t kSlotBits = 13;  // bin slots < kResMaxParticles = 2^13
constexpr uint32_t kSlotMask = (1u << kSlotBits) - 1u;
constexpr int kResPer = (int)((kResMaxParticles + kResThreads - 1) / kResThreads);  // slots per thread
constexpr int kEntWords = (kResPer + 3) / 4;  // a thread's slots' entries, 8 bits each
// Steps on which at most this many particles of a bin changed cell re-sort
// the bin incrementally; more take the full block sort.
constexpr uint32_t kResMaxMovers = 32;
static_assert(kResMaxParticles == (1u << kSlotBits), "slot field of the sort values");
static_assert(kResMaxCells <= (1u << kSlotBits), "cell field of the sort values");
static_assert(kResWarps <= 32 && kResThreads % 32 == 0,
              "the block scan is one warp over the warps' totals");
static_assert(kResPer <= 32, "a thread's moved slots are one 32-bit mask");

inline __host__ __device__ uint32_t round64(uint32_t n) { return (n + 63u) & ~63u; }

// The block's global scratch: the state stashed by the sort, the collide's
// results, and the angle, mass and id of every slot (two sets: the sort
// gathers from one into the other).  Arrays of nb (a multiple of 64) words
// or pairs, addressed from one base so that few registers hold them.
struct Work {
    char* base;
    uint32_t nb;
    __device__ __forceinline__ float2* stashPos() const { return reinterpret_cast<float2*>(base); }
    __device__ __forceinline__ float2* stashVel() const {
        return reinterpret_cast<float2*>(base + 8ull * nb);
    }
    __device__ __forceinline__ float2* F() const {
        return reinterpret_cast<float2*>(base + 16ull * nb);
    }
    __device__ __forceinline__ float* stashOm() const {
        return reinterpret_cast<float*>(base + 24ull * nb);
    }
    __device__ __forceinline__ float* stashRad() const {
        return reinterpret_cast<float*>(base + 28ull * nb);
    }
    __device__ __forceinline__ float* M() const { return reinterpret_cast<float*>(base + 32ull * nb); }
    __device__ __forceinline__ float* Pr() const { return reinterpret_cast<float*>(base + 36ull * nb); }
    __device__ __forceinline__ float* theta(int k) const {
        return reinterpret_cast<float*>(base + (40ull + 12ull * k) * nb);
    }
    __device__ __forceinline__ float* mass(int k) const {
        return reinterpret_cast<float*>(base + (44ull + 12ull * k) * nb);
    }
    __device__ __forceinline__ uint32_t* id(int k) const {
        return reinterpret_cast<uint32_t*>(base + (48ull + 12ull * k) * nb);
    }
    // the bin cell of every slot after the last integrate
    __device__ __forceinline__ uint32_t* key() const {
        return reinterpret_cast<uint32_t*>(base + 64ull * nb);
    }
};

__host__ __device__ inline size_t work_bytes_per_block(uint32_t maxN) {
    return (size_t)68 * round64(maxN);
}

// Shared memory of a block: positions, velocities, spins, radii (nb each),
// the first-particle array (round64(maxC + 1) words), the bin's entries and
// the scan words.  The sort's two value arrays alias the positions, which
// the sort has stashed first.
__host__ __device__ inline size_t smem_bytes(uint32_t maxN, uint32_t maxC) {
    const size_t nb = round64(maxN);
    return 24 * nb + 4 * (size_t)round64(maxC + 1) + sizeof(ResEntry) * kResMaxEntries +
           4 * (2 * kResWarps + 4) + sizeof(uint4) * kResMaxMovers;
}

extern __shared__ __align__(16) unsigned char smraw[];

struct Smem {
    uint32_t nb, nc;  // particle and cell capacity of the arrays
    __device__ __forceinline__ float2* pos() const { return reinterpret_cast<float2*>(smraw); }
    __device__ __forceinline__ float2* vel() const {
        return reinterpret_cast<float2*>(smraw + 8u * nb);
    }
    __device__ __forceinline__ float* omega() const {
        return reinterpret_cast<float*>(smraw + 16u * nb);
    }
    __device__ __forceinline__ float* radius() const {
        return reinterpret_cast<float*>(smraw + 20u * nb);
    }
    __device__ __forceinline__ uint32_t* first() const {
        return reinterpret_cast<uint32_t*>(smraw + 24u * nb);
    }
    __device__ __forceinline__ ResEntry* ent() const {
        return reinterpret_cast<ResEntry*>(smraw + 24u * nb + 4u * nc);
    }
    __device__ __forceinline__ uint32_t* scan() const {
        return reinterpret_cast<uint32_t*>(smraw + 24u * nb + 4u * nc +
                                           (uint32_t)sizeof(ResEntry) * kResMaxEntries);
    }
    // (slot, cell before, cell after) of the particles that changed cell
    __device__ __forceinline__ uint4* movers() const {
        return reinterpret_cast<uint4*>(smraw + 24u * nb + 4u * nc +
                                        (uint32_t)sizeof(ResEntry) * kResMaxEntries +
                                        4u * (2u * kResWarps + 4u));
    }
    __device__ __forceinline__ uint32_t* sortA() const { return reinterpret_cast<uint32_t*>(smraw); }
    __device__ __forceinline__ uint32_t* sortB() const {
        return reinterpret_cast<uint32_t*>(smraw) + nb;
    }
};

// The particle's cell in its specimen's grid, wrapped (calcGridPos +
// calcGridHash, particles_kernel.cuh:114-130; grid_pos_fast gives the
// reference's quotient bit for bit).
__device__ __forceinline__ uint32_t local_cell(const KParams& P, float2 p) {
    const int2 g = grid_pos_fast(P, p);
    return (uint32_t)(g.y & (int)(P.gy - 1u)) * P.gx + (uint32_t)(g.x & (int)(P.gx - 1u));
}

// Entry of a bin slot: the last entry whose first slot is <= i.
__device__ __forceinline__ uint32_t entry_of(const ResEntry* ent, uint32_t count, uint32_t i) {
    uint32_t lo = 0, hi = count;  // ent[lo].slot <= i < ent[hi].slot
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (ent[mid].slot <= i) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Stable sort of the n values (cell << kSlotBits | slot) in `a`, by their
// cell bits: one LSD pass per cell bit on which the values differ
// (`differ`).  Lane l of warp w holds elements w * 32 * per + k * 32 + l, so
// each warp's elements are one contiguous run and its ballots give the
// ranks.  Returns the array holding the sorted values (a or b).
template <int THREADS>
__device__ uint32_t* block_sort(uint32_t* a, uint32_t* b, uint32_t n, uint32_t differ,
                                uint32_t* scan) {
    constexpr int kWarps = THREADS / 32;
    constexpr int kPer = (int)((kResMaxParticles + THREADS - 1) / THREADS);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t per = (n + THREADS - 1u) / THREADS;
    const uint32_t wbase = (uint32_t)warp * 32u * per;
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll 1
    for (uint32_t bit = kSlotBits; bit < 2 * kSlotBits; ++bit) {
        if (!((differ >> bit) & 1u)) continue;  // every value agrees here: the pass is the identity
        uint32_t v[kPer];
        unsigned zm[kPer];
        uint32_t zeros = 0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            v[k] = 0u;
            zm[k] = 0u;
            if ((uint32_t)k < per) {
                const uint32_t e = wbase + (uint32_t)k * 32u + (uint32_t)lane;
                const bool ok = e < n;
                if (ok) v[k] = a[e];
                zm[k] = __ballot_sync(0xffffffffu, ok && !((v[k] >> bit) & 1u));
                zeros += (uint32_t)__popc(zm[k]);
            }
        }
        if (lane == 0) scan[warp] = zeros;
        __syncthreads();
        if (warp == 0) {
            uint32_t x = lane < kWarps ? scan[lane] : 0u;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
                if (lane >= d) x += y;
            }
            if (lane < kWarps) scan[kWarps + lane] = x;  // inclusive
        }
        __syncthreads();
        const uint32_t total0 = scan[2 * kWarps - 1];
        const uint32_t zBefore = warp ? scan[kWarps + warp - 1] : 0u;
        const uint32_t oBefore = min(n, wbase) - zBefore;
        uint32_t zr = 0, orr = 0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            if ((uint32_t)k < per) {
                const uint32_t e = wbase + (uint32_t)k * 32u + (uint32_t)lane;
                const bool ok = e < n;
                const unsigned z = zm[k];
                const unsigned o = __ballot_sync(0xffffffffu, ok) & ~z;
                if (ok) {
                    const uint32_t dst = ((z >> lane) & 1u)
                                             ? zBefore + zr + (uint32_t)__popc(z & lt)
                                             : total0 + oBefore + orr + (uint32_t)__popc(o & lt);
                    b[dst] = v[k];
                }
                zr += (uint32_t)__popc(z);
                orr += (uint32_t)__popc(o);
            }
        }
        uint32_t* t = a;
        a = b;
        b = t;
        __syncthreads();  // the pass is complete before the next one reads it
    }
    return a;
}


// The movers of the last step, (slot, cell before, cell after) -- at most
// kResMaxMovers of them -- ranked by one warp (warp 0 calls this) into four
// sorted arrays of ms (kResMaxMovers words each): their slots; their cells
// after with their slots, in (cell, slot) order; their cells before.  `src`
// may be ms itself (the entries are read into registers first); from
// global memory (fromGlobal) it is read through L2.
__device__ void rank_movers(const uint4* src, bool fromGlobal, uint32_t nm, uint32_t* ms) {
    const uint32_t lane = threadIdx.x & 31u;
    const bool ok = lane < nm;
    uint4 e = make_uint4(0u, 0u, 0u, 0u);
    if (ok) e = fromGlobal ? __ldcg(src + lane) : src[lane];
    __syncwarp();
    uint32_t rs = 0u, rn = 0u, ro = 0u;
#pragma unroll 4
    for (uint32_t q = 0; q < nm; ++q) {
        const uint32_t x = __shfl_sync(0xffffffffu, e.x, (int)q);
        const uint32_t y = __shfl_sync(0xffffffffu, e.y, (int)q);
        const uint32_t z = __shfl_sync(0xffffffffu, e.z, (int)q);
        rs += x < e.x ? 1u : 0u;
        rn += (z < e.z || (z == e.z && x < e.x)) ? 1u : 0u;
        ro += (y < e.y || (y == e.y && x < e.x)) ? 1u : 0u;
    }
    if (ok) {
        ms[rs] = e.x;
        ms[kResMaxMovers + rn] = e.z;
        ms[2 * kResMaxMovers + rn] = e.x;
        ms[3 * kResMaxMovers + ro] = e.y;
    }
}

// Entries of the sorted a[0, n) below v.
__device__ __forceinline__ uint32_t count_below(const uint32_t* a, uint32_t n, uint32_t v) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1u;
        else hi = mid;
    }
    return lo;
}

// A slot's place in the new stable order by cell, from the ranked movers
// (rank_movers) and the old first-particle array: a stayer moves down by
// the movers before it and up by the movers placed before it; a mover goes
// after the stayers of lower cells and of its new cell that came before it
// in the old order, then after the movers placed before it.
__device__ __forceinline__ uint32_t incremental_dest(const uint32_t* ms, uint32_t nm,
                                                     const uint32_t* first, uint32_t i,
                                                     uint32_t key) {
    const uint32_t* slots = ms;
    const uint32_t* newCell = ms + kResMaxMovers;
    const uint32_t* newSlot = ms + 2 * kResMaxMovers;
    const uint32_t rb = count_below(slots, nm, i);
    const bool isMover = rb < nm && slots[rb] == i;
    uint32_t lo = 0, hi = nm;  // movers placed before (key, i)
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (newCell[mid] < key || (newCell[mid] == key && newSlot[mid] < i)) lo = mid + 1u;
        else hi = mid;
    }
    if (!isMover) return i - rb + lo;
    const uint32_t q = min(max(i, first[key]), first[key + 1u]);
    return q - count_below(slots, nm, q) + lo;
}

// Change of cell c's first slot: the movers now below c less those that were.
__device__ __forceinline__ int first_shift(const uint32_t* ms, uint32_t nm, uint32_t c) {
    return (int)count_below(ms + kResMaxMovers, nm, c) -
           (int)count_below(ms + 3 * kResMaxMovers, nm, c);
}

// First index of the sorted values whose cell is >= c.
__device__ __forceinline__ uint32_t lower_cell(const uint32_t* v, uint32_t n, uint32_t c) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((v[mid] >> kSlotBits) < c) lo = mid + 1u;
        else hi = mid;
    }
    return lo;
}

// Forces on particle i, in cell `local` of its specimen's grid, from its
// 3 x 3 cells, in the reference's order; the neighbours' fields from shared
// memory.  With culling (the specimen's
// cells wider than 2 rmax and the particle inside the box by the margin) a
// column or row of cells farther than r + rmax is skipped: it holds no
// contact, and its subtotal would be +0.
__device__ __forceinline__ void res_collide(const KParams& P, uint32_t cellOff, uint32_t local,
                                            uint32_t i, float2 p, float2 v, float w, float r,
                                            const Smem& S, float2& force, float& moment,
                                            float& pr) {
    force = make_float2(0.0f, 0.0f);
    moment = 0.0f;
    pr = 0.0f;
    // the particle's (wrapped) cell, from its cell index in the specimen's grid
    const int gx = (int)(local & (P.gx - 1u)), gy = (int)(local >> P.log2gx);
    int y0 = -1, y1 = 1, x0 = -1, x1 = 1;
    if (P.cull && p.x > P.cullMargin && p.x < P.Lx - P.cullMargin && p.y > P.cullMargin &&
        p.y < P.Ly - P.cullMargin) {
        const float reach = (r + P.rmax) * 1.0001f + P.cullMargin;
        const float X0 = (float)gx * P.cellW, Y0 = (float)gy * P.cellH;
        if (p.x - X0 > reach) x0 = 0;
        if (X0 + P.cellW - p.x > reach) x1 = 0;
        if (p.y - Y0 > reach) y0 = 0;
        if (Y0 + P.cellH - p.y > reach) y1 = 0;
    }
    const int mx = (int)(P.gx - 1u), my = (int)(P.gy - 1u);
    // rmax bounds every radius of the batch (INFINITY when unknown): a superset
    // of the exact test below, cd <= r + rmax in float as in reals
    const float rr = r + P.rmax;
    const float reach2 = rr * rr * 1.000002f;
#pragma unroll 1
    for (int dy = y0; dy <= y1; ++dy) {
        const uint32_t row = cellOff + (uint32_t)((gy + dy) & my) * P.gx;
#pragma unroll 1
        for (int dx = x0; dx <= x1; ++dx) {
            const uint32_t h = row + (uint32_t)((gx + dx) & mx);
            const uint32_t a = S.first()[h], b = S.first()[h + 1];
            float2 fc = make_float2(0.0f, 0.0f);
#pragma unroll 1
            for (uint32_t j = a; j < b; ++j) {
                const float2 pj = S.pos()[j];
                const float ax = pj.x - p.x, ay = pj.y - p.y;
                const float d2 = ax * ax + ay * ay;
                // beyond (r + rmax)^2 (1 + 2e-6) no radius can reach: the
                // radius is read for the near candidates only
                if (d2 > reach2) continue;
                const float rj = S.radius()[j];
                const float cd = r + rj;
                // d2 > cd^2 (1 + 2e-6) implies sqrtf(d2) >= cd: no contact
                if (j != i && d2 <= cd * cd * 1.000002f && sqrtf(d2) < cd) {
                    const float2 f = pair_force(p, pj, v, S.vel()[j], w, S.omega()[j], r, rj,
                                                P.pair[0], P.dt, moment, pr);
                    fc.x += f.x;
                    fc.y += f.y;
                }
            }
            force.x += fc.x;
            force.y += fc.y;
        }
    }
}


__global__ void __launch_bounds__(kResThreads, 1)
resident_kernel(const KParams* __restrict__ table, const ResBin* __restrict__ bins,
                uint32_t numBins, const ResEntry* __restrict__ entries,
                uint32_t* __restrict__ queue, uint32_t maxN, uint32_t maxC, char* workBase,
                ResIO io, uint32_t nTotal, uint32_t nsteps, uint32_t* __restrict__ errFlag) {
    __shared__ uint32_t sBin;
    __shared__ uint32_t sMovers;  // particles that changed cell in the last step
    const Smem S{round64(maxN), round64(maxC + 1)};
    const Work W{workBase + work_bytes_per_block(maxN) * blockIdx.x, round64(maxN)};
    const uint32_t tid = threadIdx.x;
#pragma unroll 1
    for (;;) {
        __syncthreads();  // the previous bin is written back
        if (tid == 0) sBin = atomicAdd(queue, 1u);
        __syncthreads();
        const uint32_t bi = sBin;
        if (bi >= numBins) break;
        const ResBin bin = bins[bi];
        const uint32_t n = bin.n, ne = bin.count;
        if (tid < ne) S.ent()[tid] = entries[bin.first + tid];
        __syncthreads();
        // the bin's state: each specimen's slots of the batch into its slots
        // of the bin
#pragma unroll 1
        for (uint32_t e = 0; e < ne; ++e) {
            const ResEntry E = S.ent()[e];
#pragma unroll 1
            for (uint32_t j = tid; j < E.n; j += kResThreads) {
                const uint32_t s = E.slot + j, g = E.gslot + j;
                S.pos()[s] = io.pos[g];
                S.vel()[s] = io.vel[g];
                S.omega()[s] = io.omega[g];
                S.radius()[s] = io.radius[g];
                W.theta(0)[s] = io.theta[g];
                W.mass(0)[s] = io.mass[g];
                W.id(0)[s] = io.id[g];
            }
        }
        // the entry of each slot this thread owns (slots tid + k * 1024),
        // 8 bits each
        const uint32_t per = (n + kResThreads - 1u) / kResThreads;
        uint32_t entPack[kEntWords];
#pragma unroll
        for (int w = 0; w < kEntWords; ++w) entPack[w] = 0u;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kResPer; ++k) {
            const uint32_t i = tid + (uint32_t)k * kResThreads;
            if ((uint32_t)k < per && i < n)
                entPack[k >> 2] |= entry_of(S.ent(), ne, i) << ((k & 3) * 8);
        }
        int buf = 0;
        bool needSort = true, fullSort = true;  // a bin's first sort is a full sort
        if (tid == 0) sMovers = 0u;
#pragma unroll 1
        for (uint32_t step = 0; step < nsteps; ++step) {
            if (needSort && !fullSort && sMovers <= kResMaxMovers) {
                // ---- incremental sort: the few particles that changed cell
                // move to their places in the stable order by cell, the others
                // keep their order (the same permutation as the full sort)
                const uint32_t nm = sMovers;
                uint32_t* __restrict__ first = S.first();
                uint32_t* ms = reinterpret_cast<uint32_t*>(S.movers());
                if (tid < 32) rank_movers(S.movers(), false, nm, ms);
                __syncthreads();
                uint32_t moved = 0u;  // bit k: owned slot k changes
#pragma unroll 1
                for (int k = 0; k < kResPer; ++k) {
                    const uint32_t i = tid + (uint32_t)k * kResThreads;
                    if ((uint32_t)k >= per || i >= n) break;
                    const uint32_t key = W.key()[i];  // the cell after the last integrate
                    const uint32_t dst = incremental_dest(ms, nm, first, i, key);
                    if (dst != i) {
                        moved |= 1u << k;
                        W.stashPos()[dst] = S.pos()[i];
                        W.stashVel()[dst] = S.vel()[i];
                        W.stashOm()[dst] = S.omega()[i];
                        W.stashRad()[dst] = S.radius()[i];
                        W.F()[dst] = make_float2(W.theta(buf)[i], W.mass(buf)[i]);
                        reinterpret_cast<uint32_t*>(W.M())[dst] = W.id(buf)[i];
                        reinterpret_cast<uint32_t*>(W.Pr())[dst] = key;
                    }
                }
                __syncthreads();  // every destination stashed; the old first array read
                // the slots that change take what was stashed for them (a
                // permutation: the slots that receive are the slots that give)
#pragma unroll 1
                for (int k = 0; k < kResPer; ++k) {
                    if (!((moved >> k) & 1u)) continue;
                    const uint32_t i = tid + (uint32_t)k * kResThreads;
                    S.pos()[i] = W.stashPos()[i];
                    S.vel()[i] = W.stashVel()[i];
                    S.omega()[i] = W.stashOm()[i];
                    S.radius()[i] = W.stashRad()[i];
                    const float2 tm = W.F()[i];
                    W.theta(buf)[i] = tm.x;
                    W.mass(buf)[i] = tm.y;
                    W.id(buf)[i] = reinterpret_cast<const uint32_t*>(W.M())[i];
                    W.key()[i] = reinterpret_cast<const uint32_t*>(W.Pr())[i];
                }
                // first slot of every cell: one more for every mover that now
                // comes before the cell, one fewer for every mover that did
#pragma unroll 1
                for (uint32_t c = tid; c <= bin.cells; c += kResThreads)
                    first[c] = (uint32_t)((int)first[c] + first_shift(ms, nm, c));
                __syncthreads();
                if (tid == 0) sMovers = 0u;
            } else if (needSort) {
                // ---- sort.  The state is stashed first, so that the value
                // arrays may overwrite the positions; the values (cell << 13 |
                // slot) are then made from the stashed positions.
#pragma unroll 1
                for (int k = 0; k < kResPer; ++k) {
                    const uint32_t i = tid + (uint32_t)k * kResThreads;
                    if ((uint32_t)k >= per || i >= n) break;
                    W.stashPos()[i] = S.pos()[i];
                    W.stashVel()[i] = S.vel()[i];
                    W.stashOm()[i] = S.omega()[i];
                    W.stashRad()[i] = S.radius()[i];
                }
                if (tid == 0) {
                    S.scan()[2 * kResWarps] = 0u;
                    S.scan()[2 * kResWarps + 1] = 0xffffffffu;
                }
                __syncthreads();  // stash complete, words initialised
                uint32_t orv = 0u, andv = 0xffffffffu;
#pragma unroll 1
                for (int k = 0; k < kResPer; ++k) {
                    const uint32_t i = tid + (uint32_t)k * kResThreads;
                    if ((uint32_t)k >= per || i >= n) break;
                    const ResEntry& E = S.ent()[(entPack[k >> 2] >> ((k & 3) * 8)) & 0xffu];
                    const uint32_t v =
                        ((E.cellOff + local_cell(table[E.spec], W.stashPos()[i])) << kSlotBits) | i;
                    S.sortA()[i] = v;
                    orv |= v;
                    andv &= v;
                }
                orv = __reduce_or_sync(0xffffffffu, orv);
                andv = __reduce_and_sync(0xffffffffu, andv);
                if ((tid & 31) == 0) {
                    atomicOr(&S.scan()[2 * kResWarps], orv);
                    atomicAnd(&S.scan()[2 * kResWarps + 1], andv);
                }
                __syncthreads();
                // the cell bits on which the values differ (the passes use
                // other scan words)
                const uint32_t differ = S.scan()[2 * kResWarps] & ~S.scan()[2 * kResWarps + 1];
                const uint32_t* sorted =
                    block_sort<kResThreads>(S.sortA(), S.sortB(), n, differ, S.scan());
                // first particle of every cell of the bin (bin.cells + 1
                // entries); each new slot's old slot to the scratch
#pragma unroll 1
                for (uint32_t c = tid; c <= bin.cells; c += kResThreads)
                    S.first()[c] = lower_cell(sorted, n, c);
                uint32_t* from = reinterpret_cast<uint32_t*>(W.M());
#pragma unroll 1
                for (int k = 0; k < kResPer; ++k) {
                    const uint32_t i = tid + (uint32_t)k * kResThreads;
                    if ((uint32_t)k >= per || i >= n) break;
                    from[i] = sorted[i] & kSlotMask;
                    W.key()[i] = sorted[i] >> kSlotBits;
                }
                __syncthreads();  // the values are read; the state arrays are free
#pragma unroll 1
                for (int k = 0; k < kResPer; ++k) {
                    const uint32_t i = tid + (uint32_t)k * kResThreads;
                    if ((uint32_t)k >= per || i >= n) break;
                    const uint32_t f = from[i];
                    S.pos()[i] = W.stashPos()[f];
                    S.vel()[i] = W.stashVel()[f];
                    S.omega()[i] = W.stashOm()[f];
                    S.radius()[i] = W.stashRad()[f];
                    W.theta(buf ^ 1)[i] = W.theta(buf)[f];
                    W.mass(buf ^ 1)[i] = W.mass(buf)[f];
                    W.id(buf ^ 1)[i] = W.id(buf)[f];
                }
                buf ^= 1;
                __syncthreads();
                if (tid == 0) sMovers = 0u;
                fullSort = false;
            }
            // ---- collide: forces from the neighbours' current state
#pragma unroll 1
            for (int k = 0; k < kResPer; ++k) {
                const uint32_t i = tid + (uint32_t)k * kResThreads;
                if ((uint32_t)k >= per || i >= n) break;
                const ResEntry& E = S.ent()[(entPack[k >> 2] >> ((k & 3) * 8)) & 0xffu];
                const KParams& P = table[E.spec];
                float2 f;
                float moment, pr;
                res_collide(P, E.cellOff, W.key()[i] - E.cellOff, i, S.pos()[i], S.vel()[i],
                            S.omega()[i], S.radius()[i], S, f, moment, pr);
                W.F()[i] = f;
                W.M()[i] = moment;
                W.Pr()[i] = pr;
            }
            __syncthreads();
            // ---- integrate in place (each thread reads and writes only its
            // own slots), then the new cell
            const bool last = step + 1u == nsteps;
            bool mover = false;
#pragma unroll 1
            for (int k = 0; k < kResPer; ++k) {
                const uint32_t i = tid + (uint32_t)k * kResThreads;
                if ((uint32_t)k >= per || i >= n) break;
                const ResEntry& E = S.ent()[(entPack[k >> 2] >> ((k & 3) * 8)) & 0xffu];
                const KParams& P = table[E.spec];
                Dyn s;
                s.p = S.pos()[i];
                s.v = S.vel()[i];
                s.w = S.omega()[i];
                s.th = W.theta(buf)[i];
                const float r = S.radius()[i];
                const float m = W.mass(buf)[i];
                const float2 f = W.F()[i];
                const float moment = W.M()[i];
                float pr = W.Pr()[i];
                const uint32_t keyBefore = W.key()[i];  // the cell this step sorted by
                // F/m and M/I as the reference divides them; without contacts
                // F and M are +0 and the quotients exactly +0 (the step
                // kernel's shortcut, the same bits)
                const bool quiet = f.x == 0.0f && f.y == 0.0f && moment == 0.0f && m > 0.0f &&
                                   m < INFINITY;
                const float two_mrr = 2.0f * m * r * r;
                float2 a;
                float al;
                if (quiet && two_mrr >= 1e-30f && two_mrr <= 1e30f) {
                    a = make_float2(0.0f, 0.0f);
                    al = 0.0f;
                } else {
                    a = make_float2(f.x / m, f.y / m);
                    al = moment / inertia_of(m, r);
                }
                integrate_one(P, s, a, al, r, m, 0u, pr);
                S.pos()[i] = s.p;
                S.vel()[i] = s.v;
                S.omega()[i] = s.w;
                W.theta(buf)[i] = s.th;
                if (!(isfinite(s.p.x) && isfinite(s.p.y))) atomicOr(errFlag, 1u);
                const uint32_t keyAfter = E.cellOff + local_cell(P, s.p);
                W.key()[i] = keyAfter;
                if (keyAfter != keyBefore) {
                    mover = true;
                    const uint32_t slot = atomicAdd(&sMovers, 1u);
                    if (slot < kResMaxMovers)
                        S.movers()[slot] = make_uint4(i, keyBefore, keyAfter, 0u);
                }
                if (last) {
                    const uint32_t g = E.gslot + (i - E.slot);
                    if (io.pressure) io.pressure[g] = pr;
                    if (io.acc) io.acc[g] = a;
                    if (io.alpha) io.alpha[g] = al;
                }
            }
            needSort = __syncthreads_or(mover) != 0;
        }
        // the bin's state back into the batch, in the order of its last sort
#pragma unroll 1
        for (uint32_t e = 0; e < ne; ++e) {
            const ResEntry E = S.ent()[e];
#pragma unroll 1
            for (uint32_t j = tid; j < E.n; j += kResThreads) {
                const uint32_t s = E.slot + j, g = E.gslot + j;
                io.pos[g] = S.pos()[s];
                io.vel[g] = S.vel()[s];
                io.omega[g] = S.omega()[s];
                io.radius[g] = S.radius()[s];
                io.theta[g] = W.theta(buf)[s];
                io.mass[g] = W.mass(buf)[s];
                const uint32_t id = W.id(buf)[s];
                io.id[g] = id;
                if (id < nTotal) io.loc[id] = g;  // ids outside 0..N-1 have no loc entry
            }
        }
    }
}


// ---------------------------------------------------------------------------
// One scene across a thread-block cluster (DEM_CTX_RESIDENT on a single
// scene of at most kResMaxParticles disks and kResMaxCells cells): the
// cluster's kClusterCtas blocks, one per multiprocessor, each hold a full
// copy of the scene's positions, velocities, spins and radii in shared
// memory, and each steps its own share of the slots.  A step is
//   sort      only after a step in which a disk changed cell: every block
//             runs the same sort (incremental or full, as above) on its own
//             copy, which gives the same permutation in every block; block 0
//             also moves the angles, masses and ids, which live in global
//             memory;
//   collide   the block's slots against its own copy;
//   integrate the block's slots, held in registers (a thread keeps its
//             slot's cell, angle and mass in registers between sorts);
//   broadcast after a cluster barrier (every copy read), each block writes
//             its slots' new positions, velocities and spins into every
//             block's copy through distributed shared memory; a second
//             cluster barrier makes them visible.
// Every block takes the same cluster barriers in the same order whatever
// its data: the sort decision reads a counter after a barrier, and no sort
// path contains a cluster barrier.  Global memory another block wrote is
// read through L2 (__ldcg).

constexpr int kClusterCtas = 8;  // blocks of a cluster (the portable size; 16 measured slower)

// Global scratch of one cluster: angles, masses, ids (two sets), the cell of
// every slot, the incremental sort's stash of those four, two mover counters
// and lists, and per block the full sort's stash and source slots.
struct CWork {
    char* base;
    uint32_t nb;
    __device__ __forceinline__ float* theta(int k) const {
        return reinterpret_cast<float*>(base + (12ull * k) * nb);
    }
    __device__ __forceinline__ float* mass(int k) const {
        return reinterpret_cast<float*>(base + (4ull + 12ull * k) * nb);
    }
    __device__ __forceinline__ uint32_t* id(int k) const {
        return reinterpret_cast<uint32_t*>(base + (8ull + 12ull * k) * nb);
    }
    __device__ __forceinline__ uint32_t* key() const {
        return reinterpret_cast<uint32_t*>(base + 24ull * nb);
    }
    __device__ __forceinline__ float2* stashTM() const {
        return reinterpret_cast<float2*>(base + 28ull * nb);
    }
    __device__ __forceinline__ uint32_t* stashId() const {
        return reinterpret_cast<uint32_t*>(base + 36ull * nb);
    }
    __device__ __forceinline__ uint32_t* stashKey() const {
        return reinterpret_cast<uint32_t*>(base + 40ull * nb);
    }
    __device__ __forceinline__ char* block(uint32_t r) const {
        return base + (44ull + 28ull * r) * nb;
    }
    __device__ __forceinline__ float2* stashPos(uint32_t r) const {
        return reinterpret_cast<float2*>(block(r));
    }
    __device__ __forceinline__ float2* stashVel(uint32_t r) const {
        return reinterpret_cast<float2*>(block(r) + 8ull * nb);
    }
    __device__ __forceinline__ float* stashOm(uint32_t r) const {
        return reinterpret_cast<float*>(block(r) + 16ull * nb);
    }
    __device__ __forceinline__ float* stashRad(uint32_t r) const {
        return reinterpret_cast<float*>(block(r) + 20ull * nb);
    }
    __device__ __forceinline__ uint32_t* from(uint32_t r) const {
        return reinterpret_cast<uint32_t*>(block(r) + 24ull * nb);
    }
    __device__ __forceinline__ uint32_t* counter() const {
        return reinterpret_cast<uint32_t*>(base + (44ull + 28ull * kClusterCtas) * nb);
    }
    __device__ __forceinline__ uint4* movers(int k) const {
        return reinterpret_cast<uint4*>(base + (44ull + 28ull * kClusterCtas) * nb + 256u) +
               k * kResMaxMovers;
    }
};

__host__ __device__ inline size_t cluster_work_bytes(uint32_t n) {
    return (44ull + 28ull * kClusterCtas) * round64(n) + 256u + 2u * 16u * kResMaxMovers;
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1)
cluster_kernel(const __grid_constant__ KParams P, ResIO io, uint32_t n, uint32_t cells,
               char* workBase, uint32_t nsteps, uint32_t* __restrict__ errFlag) {
    constexpr int kPer = (int)((kResMaxParticles + THREADS - 1) / THREADS);
    static_assert(kPer <= 32, "a thread's moved slots are one 32-bit mask");
    cg::cluster_group cl = cg::this_cluster();
    const uint32_t rank = cl.block_rank();
    const uint32_t tid = threadIdx.x;
    const Smem S{round64(n), round64(cells + 1)};
    const CWork W{workBase, round64(n)};
    // this thread's slot
    const uint32_t ctas = cl.num_blocks();
    const uint32_t share = (n + ctas - 1u) / ctas;
    const uint32_t own = rank * share + tid;
    const bool mine = tid < share && own < n;
    const uint32_t per = (n + THREADS - 1u) / THREADS;  // slots of the copy per thread
#pragma unroll 1
    for (uint32_t i = tid; i < n; i += THREADS) {
        S.pos()[i] = io.pos[i];
        S.vel()[i] = io.vel[i];
        S.omega()[i] = io.omega[i];
        S.radius()[i] = io.radius[i];
        if (rank == 0) {
            W.theta(0)[i] = io.theta[i];
            W.mass(0)[i] = io.mass[i];
            W.id(0)[i] = io.id[i];
        }
    }
    if (rank == 0 && tid < 2) W.counter()[tid] = 0u;
    int buf = 0;
    bool needSort = true, fullSort = true;
    // the own slot's cell, angle and mass, kept in registers between sorts
    uint32_t myKey = 0u;
    float myTh = 0.0f, myM = 0.0f;
    cl.sync();
#pragma unroll 1
    for (uint32_t step = 0; step < nsteps; ++step) {
        const int par = (int)(step & 1u);  // this step's movers: counter / list par
        const bool sorting = needSort;
        if (needSort) {
            const uint32_t nm = fullSort ? 0xffffffffu : __ldcg(W.counter() + (par ^ 1));
            const uint4* __restrict__ mv = W.movers(par ^ 1);
            uint32_t* __restrict__ first = S.first();
            if (nm <= kResMaxMovers) {
                // ---- incremental sort of this block's copy (as in
                // resident_kernel, over every slot of the copy)
                uint32_t* ms = reinterpret_cast<uint32_t*>(S.movers());
                if (tid < 32) rank_movers(mv, true, nm, ms);
                __syncthreads();
                uint32_t moved = 0u;
#pragma unroll 1
                for (int k = 0; k < kPer; ++k) {
                    const uint32_t i = tid + (uint32_t)k * THREADS;
                    if ((uint32_t)k >= per || i >= n) break;
                    // the slot's cell from the copy's position (the cell array
                    // in global memory is rewritten by block 0 meanwhile)
                    const uint32_t key = local_cell(P, S.pos()[i]);
                    const uint32_t dst = incremental_dest(ms, nm, first, i, key);
                    if (dst != i) {
                        moved |= 1u << k;
                        W.stashPos(rank)[dst] = S.pos()[i];
                        W.stashVel(rank)[dst] = S.vel()[i];
                        W.stashOm(rank)[dst] = S.omega()[i];
                        W.stashRad(rank)[dst] = S.radius()[i];
                        if (rank == 0) {
                            W.stashTM()[dst] = make_float2(__ldcg(W.theta(buf) + i),
                                                           __ldcg(W.mass(buf) + i));
                            W.stashId()[dst] = __ldcg(W.id(buf) + i);
                            W.stashKey()[dst] = key;
                        }
                    }
                }
                __syncthreads();
#pragma unroll 1
                for (int k = 0; k < kPer; ++k) {
                    if (!((moved >> k) & 1u)) continue;
                    const uint32_t i = tid + (uint32_t)k * THREADS;
                    S.pos()[i] = W.stashPos(rank)[i];
                    S.vel()[i] = W.stashVel(rank)[i];
                    S.omega()[i] = W.stashOm(rank)[i];
                    S.radius()[i] = W.stashRad(rank)[i];
                    if (rank == 0) {
                        const float2 tm = W.stashTM()[i];
                        W.theta(buf)[i] = tm.x;
                        W.mass(buf)[i] = tm.y;
                        W.id(buf)[i] = W.stashId()[i];
                        W.key()[i] = W.stashKey()[i];
                    }
                }
#pragma unroll 1
                for (uint32_t c = tid; c <= cells; c += THREADS)
                    first[c] = (uint32_t)((int)first[c] + first_shift(ms, nm, c));
                __syncthreads();
            } else {
                // ---- full sort of this block's copy
#pragma unroll 1
                for (uint32_t i = tid; i < n; i += THREADS) {
                    W.stashPos(rank)[i] = S.pos()[i];
                    W.stashVel(rank)[i] = S.vel()[i];
                    W.stashOm(rank)[i] = S.omega()[i];
                    W.stashRad(rank)[i] = S.radius()[i];
                }
                if (tid == 0) {
                    S.scan()[2 * (THREADS / 32)] = 0u;
                    S.scan()[2 * (THREADS / 32) + 1] = 0xffffffffu;
                }
                __syncthreads();
                uint32_t orv = 0u, andv = 0xffffffffu;
#pragma unroll 1
                for (uint32_t i = tid; i < n; i += THREADS) {
                    const uint32_t v = (local_cell(P, W.stashPos(rank)[i]) << kSlotBits) | i;
                    S.sortA()[i] = v;
                    orv |= v;
                    andv &= v;
                }
                orv = __reduce_or_sync(0xffffffffu, orv);
                andv = __reduce_and_sync(0xffffffffu, andv);
                if ((tid & 31) == 0) {
                    atomicOr(&S.scan()[2 * (THREADS / 32)], orv);
                    atomicAnd(&S.scan()[2 * (THREADS / 32) + 1], andv);
                }
                __syncthreads();
                const uint32_t differ =
                    S.scan()[2 * (THREADS / 32)] & ~S.scan()[2 * (THREADS / 32) + 1];
                const uint32_t* sorted =
                    block_sort<THREADS>(S.sortA(), S.sortB(), n, differ, S.scan());
#pragma unroll 1
                for (uint32_t c = tid; c <= cells; c += THREADS) first[c] = lower_cell(sorted, n, c);
#pragma unroll 1
                for (uint32_t i = tid; i < n; i += THREADS) {
                    W.from(rank)[i] = sorted[i] & kSlotMask;
                    if (rank == 0) W.key()[i] = sorted[i] >> kSlotBits;
                }
                __syncthreads();  // the values are read; the copy's arrays are free
#pragma unroll 1
                for (uint32_t i = tid; i < n; i += THREADS) {
                    const uint32_t f = W.from(rank)[i];
                    S.pos()[i] = W.stashPos(rank)[f];
                    S.vel()[i] = W.stashVel(rank)[f];
                    S.omega()[i] = W.stashOm(rank)[f];
                    S.radius()[i] = W.stashRad(rank)[f];
                    if (rank == 0) {
                        W.theta(buf ^ 1)[i] = __ldcg(W.theta(buf) + f);
                        W.mass(buf ^ 1)[i] = __ldcg(W.mass(buf) + f);
                        W.id(buf ^ 1)[i] = __ldcg(W.id(buf) + f);
                    }
                }
                buf ^= 1;
                __syncthreads();
            }
            fullSort = false;
        }
        cl.sync();  // every copy sorted; block 0's angles, masses, ids and cells visible
        // the previous step's mover count is consumed: it counts this step's
        // successor's movers next
        if (rank == 0 && tid == 0) W.counter()[par ^ 1] = 0u;
        if (sorting && mine) {
            // the slot now holds another disk: its cell from the copy, its
            // angle and mass from block 0's permutation
            myKey = local_cell(P, S.pos()[own]);
            myTh = __ldcg(W.theta(buf) + own);
            myM = __ldcg(W.mass(buf) + own);
        }
        const bool last = step + 1u == nsteps;
        Dyn s;
        if (mine) {
            const uint32_t keyBefore = myKey;
            float2 f;
            float moment, pr;
            s.p = S.pos()[own];
            s.v = S.vel()[own];
            s.w = S.omega()[own];
            const float r = S.radius()[own];
            res_collide(P, 0u, keyBefore, own, s.p, s.v, s.w, r, S, f, moment, pr);
            s.th = myTh;
            const float m = myM;
            const bool quiet = f.x == 0.0f && f.y == 0.0f && moment == 0.0f && m > 0.0f &&
                               m < INFINITY;
            const float two_mrr = 2.0f * m * r * r;
            float2 a;
            float al;
            if (quiet && two_mrr >= 1e-30f && two_mrr <= 1e30f) {
                a = make_float2(0.0f, 0.0f);
                al = 0.0f;
            } else {
                a = make_float2(f.x / m, f.y / m);
                al = moment / inertia_of(m, r);
            }
            integrate_one(P, s, a, al, r, m, 0u, pr);
            myTh = s.th;
            W.theta(buf)[own] = s.th;  // for block 0's permutation at the next sort
            if (!(isfinite(s.p.x) && isfinite(s.p.y))) atomicOr(errFlag, 1u);
            const uint32_t keyAfter = local_cell(P, s.p);
            myKey = keyAfter;
            if (keyAfter != keyBefore) {
                const uint32_t slot = atomicAdd(W.counter() + par, 1u);
                if (slot < kResMaxMovers)
                    W.movers(par)[slot] = make_uint4(own, keyBefore, keyAfter, 0u);
            }
            if (last) {
                if (io.pressure) io.pressure[own] = pr;
                if (io.acc) io.acc[own] = a;
                if (io.alpha) io.alpha[own] = al;
            }
        }
        // every block has read its copy (each value read was used above), so
        // the copies may be overwritten: an arrive without release semantics
        asm volatile("barrier.cluster.arrive.relaxed;\n\tbarrier.cluster.wait;" ::: "memory");
        if (mine) {
#pragma unroll 1
            for (uint32_t r = 0; r < ctas; ++r) {
                cl.map_shared_rank(S.pos(), r)[own] = s.p;
                cl.map_shared_rank(S.vel(), r)[own] = s.v;
                cl.map_shared_rank(S.omega(), r)[own] = s.w;
            }
        }
        cl.sync();  // every copy holds the new state; the mover count is final
        needSort = __ldcg(W.counter() + par) != 0u;
    }
    // this block's slots back into the scene, in the order of the last sort
    if (mine) {
        io.pos[own] = S.pos()[own];
        io.vel[own] = S.vel()[own];
        io.omega[own] = S.omega()[own];
        io.radius[own] = S.radius()[own];
        io.theta[own] = myTh;
        io.mass[own] = myM;
        const uint32_t id = __ldcg(W.id(buf) + own);
        io.id[own] = id;
        if (id < n) io.loc[id] = own;
    }
    cl.sync();  // no block leaves while another may still address its shared memory
}

}  // namespace

bool resident_plan(const std::vector<uint32_t>& partOff, const std::vector<uint32_t>& cells,
                   std::vector<ResEntry>& entries, std::vector<ResBin>& bins, uint32_t& maxN,
                   uint32_t& maxC) {
    const uint32_t ns = (uint32_t)cells.size();
    if (partOff.size() != (size_t)ns + 1u) return false;
    std::vector<uint32_t> order(ns);
    for (uint32_t s = 0; s < ns; ++s) order[s] = s;
    auto count = [&](uint32_t s) { return partOff[s + 1] - partOff[s]; };
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return count(a) > count(b); });
    struct Open {
        uint32_t n, c;
        std::vector<uint32_t> specs;
    };
    std::vector<Open> open;
    for (uint32_t s : order) {
        const uint32_t n = count(s), c = cells[s];
        if (n == 0) continue;  // nothing to step
        if (n > kResMaxParticles || c > kResMaxCells) return false;
        size_t b = 0;
        for (; b < open.size(); ++b)
            if (open[b].n + n <= kResMaxParticles && open[b].c + c <= kResMaxCells &&
                open[b].specs.size() < kResMaxEntries)
                break;
        if (b == open.size()) open.push_back(Open{0u, 0u, {}});
        open[b].n += n;
        open[b].c += c;
        open[b].specs.push_back(s);
    }
    std::stable_sort(open.begin(), open.end(),
                     [](const Open& a, const Open& b) { return a.n > b.n; });
    entries.clear();
    bins.clear();
    maxN = 0;
    maxC = 0;
    for (const Open& o : open) {
        ResBin b{(uint32_t)entries.size(), (uint32_t)o.specs.size(), o.n, o.c};
        uint32_t slot = 0, cell = 0;
        for (uint32_t s : o.specs) {
            entries.push_back(ResEntry{s, partOff[s], slot, count(s), cell, cells[s]});
            slot += count(s);
            cell += cells[s];
        }
        bins.push_back(b);
        maxN = std::max(maxN, o.n);
        maxC = std::max(maxC, o.c);
    }
    return true;
}

size_t resident_work_bytes(uint32_t maxN) { return work_bytes_per_block(maxN); }

size_t resident_smem_bytes(uint32_t maxN, uint32_t maxC) { return smem_bytes(maxN, maxC); }

int resident_blocks(uint32_t numBins, int device) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        sms <= 0)
        sms = 1;
    return (int)std::min<uint32_t>(numBins, (uint32_t)sms);
}

cudaError_t launch_resident(const KParams* table, const ResBin* bins, uint32_t numBins,
                            const ResEntry* entries, uint32_t maxN, uint32_t maxC,
                            uint32_t* queue, void* work, int blocks, ResIO io, uint32_t nTotal,
                            uint32_t nsteps, uint32_t* errFlag, cudaStream_t st) {
    if (numBins == 0 || nsteps == 0) return cudaSuccess;
    const size_t smem = smem_bytes(maxN, maxC);
    cudaError_t e = cudaFuncSetAttribute(resident_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(queue, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    resident_kernel<<<blocks, kResThreads, smem, st>>>(table, bins, numBins, entries, queue, maxN,
                                                       maxC, static_cast<char*>(work), io, nTotal,
                                                       nsteps, errFlag);
    return cudaGetLastError();
}


size_t cluster_scene_work_bytes(uint32_t n) { return cluster_work_bytes(n); }

bool cluster_scene_fits(uint32_t n, uint32_t cells) {
    return n >= 1u && n <= kResMaxParticles && cells <= kResMaxCells;
}

cudaError_t launch_cluster_scene(const KParams& P, uint32_t n, uint32_t cells, void* work,
                                 ResIO io, uint32_t nsteps, uint32_t* errFlag, cudaStream_t st) {
    if (n == 0 || nsteps == 0) return cudaSuccess;
    if (!cluster_scene_fits(n, cells)) return cudaErrorInvalidValue;
    const size_t smem = smem_bytes(n, cells);
    // a launch of `ctas` blocks of `threads`, or cudaErrorNotSupported when no
    // such cluster can be resident
    auto launch = [&](auto kernel, int threads, int ctas) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)ctas, 1, 1);
        cfg.blockDim = dim3((unsigned)threads, 1, 1);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)ctas;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        e = cudaOccupancyMaxActiveClusters(&clusters, kernel, &cfg);
        if (e != cudaSuccess || clusters < 1) {
            (void)cudaGetLastError();  // the query's error is not the caller's
            return cudaErrorNotSupported;
        }
        return cudaLaunchKernelEx(&cfg, kernel, P, io, n, cells, static_cast<char*>(work),
                                  nsteps, errFlag);
    };
    const uint32_t share = (n + (uint32_t)kClusterCtas - 1u) / (uint32_t)kClusterCtas;
    return share <= 512u ? launch(cluster_kernel<512>, 512, kClusterCtas)
                         : launch(cluster_kernel<1024>, 1024, kClusterCtas);
}

}  // namespace dem
