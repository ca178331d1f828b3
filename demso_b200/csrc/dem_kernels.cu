// DEM step kernels: hash, reorder + cell ranges, collide, integrate, and the
// fused collide/integrate/hash kernel the context's step uses.
#include "dem_kernels.cuh"

namespace dem {
namespace {

constexpr int kThreads = 256;
constexpr int kCollideThreads = 128;

inline unsigned blocks_for(uint32_t n, int t) { return (unsigned)((n + (uint32_t)t - 1u) / (uint32_t)t); }

// particles_kernel.cuh:133-151
__global__ void __launch_bounds__(kThreads)
calc_hash_kernel(KParams P, const float2* __restrict__ pos, uint32_t* __restrict__ hash,
                 uint32_t* __restrict__ index, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int2 g = grid_pos(P, pos[i]);
    hash[i] = grid_hash(P, g.x, g.y);
    if (index) index[i] = i;
}

// particles_kernel.cuh:156-233.  A cell starts where the sorted hash differs
// from its predecessor; the predecessor's cell ends there.  The reference
// stages hashes in shared memory; here the neighbour comes from the next lane
// by shuffle and only lane 0 reads hash[i-1] (an L1 hit).
template <bool TYPED>
__global__ void __launch_bounds__(kThreads)
reorder_kernel(uint32_t* __restrict__ cellStart, uint32_t* __restrict__ cellEnd, DynSet s,
               StatSet sS, uint32_t* __restrict__ sLoc, const uint32_t* __restrict__ hash,
               const uint32_t* __restrict__ index, DynSet o, StatSet oS, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    const uint32_t h = valid ? hash[i] : 0u;
    uint32_t hp = __shfl_up_sync(0xffffffffu, h, 1);
    if ((threadIdx.x & 31) == 0 && valid && i > 0) hp = hash[i - 1];
    if (!valid) return;
    if (i == 0 || h != hp) {
        cellStart[h] = i;
        if (i > 0) cellEnd[hp] = i;
    }
    if (i == n - 1) cellEnd[h] = i + 1;
    const uint32_t src = index[i];
    s.pos[i] = o.pos[src];
    s.vel[i] = o.vel[src];
    s.theta[i] = o.theta[src];
    s.omega[i] = o.omega[src];
    sS.radius[i] = oS.radius[src];
    sS.mass[i] = oS.mass[src];
    const uint32_t id = oS.id[src];
    sS.id[i] = id;
    sLoc[id] = i;
    if (TYPED) sS.type[i] = oS.type[src];
}

// Sum of the forces on particle i from its 3x3 cell neighbourhood,
// particles_kernel.cuh:459-549 (collideD) with collideCell (:346-385): cells
// y-outer, x-inner, particles in ascending sorted index, each cell's
// subtotal added to the running force.  Wrapping makes a 1- or 2-wide grid
// visit the same cell more than once, exactly as the reference does.
template <bool TYPED, bool ATTRACT>
__device__ __forceinline__ void collide_one(const KParams& P, uint32_t i, float2 p, float2 v,
                                            float w, float r, uint32_t mat,
                                            const float2* __restrict__ pos,
                                            const float2* __restrict__ vel,
                                            const float* __restrict__ omega,
                                            const float* __restrict__ radius,
                                            const uint32_t* __restrict__ type,
                                            const uint32_t* __restrict__ cellStart,
                                            const uint32_t* __restrict__ cellEnd, float2& force,
                                            float& moment, float& pr) {
    const int2 g = grid_pos(P, p);
    force = make_float2(0.0f, 0.0f);
    moment = 0.0f;
    pr = 0.0f;
    const float4 pc0 = P.pair[0];
#pragma unroll 1
    for (int dy = -1; dy <= 1; ++dy) {
#pragma unroll 1
        for (int dx = -1; dx <= 1; ++dx) {
            const uint32_t h = grid_hash(P, g.x + dx, g.y + dy);
            const uint32_t start = __ldg(cellStart + h);
            float2 fc = make_float2(0.0f, 0.0f);
            if (start != kEmptyCell) {
                const uint32_t end = __ldg(cellEnd + h);
#pragma unroll 1
                for (uint32_t j = start; j < end; ++j) {
                    if (j == i) continue;
                    const float2 pj = __ldg(pos + j);
                    const float rj = __ldg(radius + j);
                    uint32_t mj = 0;
                    float4 pc = pc0;
                    if (TYPED) {
                        mj = __ldg(type + j);
                        pc = P.pair[mat * P.nmat + mj];
                    }
                    // contact test first; velocity/omega of j only for contacts
                    const float relx = pj.x - p.x, rely = pj.y - p.y;
                    const float dist = len2(relx, rely);
                    if (dist < r + rj) {
                        const float2 f = pair_force(p, pj, v, __ldg(vel + j), w, __ldg(omega + j),
                                                    r, rj, pc, P.dt, moment, pr);
                        fc.x += f.x;
                        fc.y += f.y;
                    }
                    if (ATTRACT) {
                        const float2 f = pair_attract(p, pj, r, rj, P.at[mat], P.at[mj], pr);
                        fc.x += f.x;
                        fc.y += f.y;
                    }
                }
            }
            force.x += fc.x;
            force.y += fc.y;
        }
    }
}

template <bool TYPED, bool ATTRACT>
__global__ void __launch_bounds__(kCollideThreads)
collide_kernel(KParams P, const float2* __restrict__ pos, const float2* __restrict__ vel,
               const float* __restrict__ omega, const float* __restrict__ radius,
               const float* __restrict__ mass, const uint32_t* __restrict__ type,
               const uint32_t* __restrict__ cellStart, const uint32_t* __restrict__ cellEnd,
               float2* __restrict__ acc, float* __restrict__ alpha, float* __restrict__ pressure,
               uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float2 p = pos[i];
    const float2 v = vel[i];
    const float w = omega[i];
    const float r = radius[i];
    const uint32_t mat = TYPED ? type[i] : 0u;
    float2 f;
    float moment, pr;
    collide_one<TYPED, ATTRACT>(P, i, p, v, w, r, mat, pos, vel, omega, radius, type, cellStart,
                                cellEnd, f, moment, pr);
    const float m = mass[i];
    acc[i] = make_float2(f.x / m, f.y / m);
    alpha[i] = moment / inertia_of(m, r);
    if (pressure) pressure[i] = pr;
}

template <bool TYPED>
__global__ void __launch_bounds__(kThreads)
integrate_kernel(KParams P, float2* __restrict__ pos, float2* __restrict__ vel,
                 const float2* __restrict__ acc, float* __restrict__ theta,
                 float* __restrict__ omega, const float* __restrict__ alpha,
                 const uint32_t* __restrict__ type, const float* __restrict__ radius,
                 const float* __restrict__ mass, float* __restrict__ pressure, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Dyn s;
    s.p = pos[i];
    s.v = vel[i];
    s.th = theta[i];
    s.w = omega[i];
    float pr = pressure ? pressure[i] : 0.0f;
    const uint32_t mat = TYPED ? type[i] : 0u;
    integrate_one(P, s, acc[i], alpha[i], radius[i], mass[i], mat, pr);
    pos[i] = s.p;
    vel[i] = s.v;
    theta[i] = s.th;
    omega[i] = s.w;
    if (pressure) pressure[i] = pr;
}

// collideD + integrateSystemD + calcHashD of the next step for one particle.
// The acceleration stays in registers instead of a round trip through HBM;
// the arithmetic is the same expressions in the same order.
template <bool TYPED, bool ATTRACT>
__global__ void __launch_bounds__(kCollideThreads)
step_kernel(KParams P, DynSet in, StatSet inS, const uint32_t* __restrict__ cellStart,
            const uint32_t* __restrict__ cellEnd, DynSet out, uint32_t* __restrict__ nextHash,
            float* __restrict__ pressure, float2* __restrict__ acc, float* __restrict__ alpha,
            uint32_t* __restrict__ errFlag, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Dyn s;
    s.p = in.pos[i];
    s.v = in.vel[i];
    s.w = in.omega[i];
    const float r = inS.radius[i];
    const uint32_t mat = TYPED ? inS.type[i] : 0u;
    float2 f;
    float moment, pr;
    collide_one<TYPED, ATTRACT>(P, i, s.p, s.v, s.w, r, mat, in.pos, in.vel, in.omega, inS.radius,
                                inS.type, cellStart, cellEnd, f, moment, pr);
    const float m = inS.mass[i];
    const float2 a = make_float2(f.x / m, f.y / m);
    const float al = moment / inertia_of(m, r);
    if (acc) acc[i] = a;
    if (alpha) alpha[i] = al;
    s.th = in.theta[i];
    integrate_one(P, s, a, al, r, m, mat, pr);
    out.pos[i] = s.p;
    out.vel[i] = s.v;
    out.theta[i] = s.th;
    out.omega[i] = s.w;
    if (pressure) pressure[i] = pr;
    const int2 g = grid_pos(P, s.p);
    nextHash[i] = grid_hash(P, g.x, g.y);
    if (!(isfinite(s.p.x) && isfinite(s.p.y))) atomicOr(errFlag, 1u);
}

// One row of the reference's followed-particle output per id
// (functions.cu:630-654): id, type, pos, vel, acc, theta, omega, alpha, pressure.
__global__ void followed_kernel(FollowIds f, const uint32_t* __restrict__ loc, DynSet d, StatSet s,
                                const float2* __restrict__ acc, const float* __restrict__ alpha,
                                const float* __restrict__ pressure, float* __restrict__ rows) {
    const uint32_t k = threadIdx.x;
    if (k >= f.count) return;
    const uint32_t i = loc[f.id[k]];
    float* r = rows + 12 * k;
    r[0] = __uint_as_float(s.id[i]);
    r[1] = __uint_as_float(s.type ? s.type[i] : 0u);
    const float2 p = d.pos[i], v = d.vel[i];
    r[2] = p.x;
    r[3] = p.y;
    r[4] = v.x;
    r[5] = v.y;
    const float2 a = acc ? acc[i] : make_float2(0.0f, 0.0f);
    r[6] = a.x;
    r[7] = a.y;
    r[8] = d.theta[i];
    r[9] = d.omega[i];
    r[10] = alpha ? alpha[i] : 0.0f;
    r[11] = pressure ? pressure[i] : 0.0f;
}

bool has_attraction(const KParams& P) {
    for (uint32_t m = 0; m < P.nmat; ++m)
        if (P.at[m] != 0.0f) return true;
    return false;
}

}  // namespace

cudaError_t launch_followed(const FollowIds& f, const uint32_t* loc, DynSet d, StatSet s,
                            const float2* acc, const float* alpha, const float* pressure,
                            float* rows, cudaStream_t st) {
    followed_kernel<<<1, kFollowBatch, 0, st>>>(f, loc, d, s, acc, alpha, pressure, rows);
    return cudaGetLastError();
}

cudaError_t launch_calc_hash(const KParams& P, const float2* pos, uint32_t* hash, uint32_t* index,
                             uint32_t n, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    calc_hash_kernel<<<blocks_for(n, kThreads), kThreads, 0, st>>>(P, pos, hash, index, n);
    return cudaGetLastError();
}

cudaError_t launch_reorder(const KParams& P, uint32_t* cellStart, uint32_t* cellEnd,
                           DynSet sorted, StatSet sortedS, uint32_t* sortedLoc,
                           const uint32_t* hash, const uint32_t* index, DynSet old, StatSet oldS,
                           uint32_t n, uint32_t numCells, bool clearCells, cudaStream_t st,
                           int* launches) {
    (void)P;
    if (clearCells) {
        cudaError_t e = cudaMemsetAsync(cellStart, 0xff, sizeof(uint32_t) * (size_t)numCells, st);
        if (e != cudaSuccess) return e;
    }
    if (n == 0) return cudaSuccess;
    if (sortedS.type && oldS.type)
        reorder_kernel<true><<<blocks_for(n, kThreads), kThreads, 0, st>>>(
            cellStart, cellEnd, sorted, sortedS, sortedLoc, hash, index, old, oldS, n);
    else
        reorder_kernel<false><<<blocks_for(n, kThreads), kThreads, 0, st>>>(
            cellStart, cellEnd, sorted, sortedS, sortedLoc, hash, index, old, oldS, n);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t launch_collide(const KParams& P, const float2* pos, const float2* vel,
                           const float* omega, const float* radius, const float* mass,
                           const uint32_t* type, const uint32_t* cellStart,
                           const uint32_t* cellEnd, float2* acc, float* alpha, float* pressure,
                           uint32_t n, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const bool typed = type != nullptr && P.nmat > 1;
    const bool attract = has_attraction(P);
    const unsigned b = blocks_for(n, kCollideThreads);
#define DEM_COLLIDE(T, A)                                                                     \
    collide_kernel<T, A><<<b, kCollideThreads, 0, st>>>(P, pos, vel, omega, radius, mass, type, \
                                                        cellStart, cellEnd, acc, alpha,        \
                                                        pressure, n)
    if (typed) {
        if (attract) DEM_COLLIDE(true, true); else DEM_COLLIDE(true, false);
    } else {
        if (attract) DEM_COLLIDE(false, true); else DEM_COLLIDE(false, false);
    }
#undef DEM_COLLIDE
    return cudaGetLastError();
}

cudaError_t launch_integrate(const KParams& P, float2* pos, float2* vel, const float2* acc,
                             float* theta, float* omega, const float* alpha, const uint32_t* type,
                             const float* radius, const float* mass, float* pressure, uint32_t n,
                             cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const unsigned b = blocks_for(n, kThreads);
    if (type != nullptr && P.nmat > 1)
        integrate_kernel<true><<<b, kThreads, 0, st>>>(P, pos, vel, acc, theta, omega, alpha, type,
                                                       radius, mass, pressure, n);
    else
        integrate_kernel<false><<<b, kThreads, 0, st>>>(P, pos, vel, acc, theta, omega, alpha,
                                                        type, radius, mass, pressure, n);
    return cudaGetLastError();
}

cudaError_t launch_step(const KParams& P, DynSet in, StatSet inS, const uint32_t* cellStart,
                        const uint32_t* cellEnd, DynSet out, uint32_t* nextHash, float* pressure,
                        float2* acc, float* alpha, uint32_t* errFlag, uint32_t n,
                        cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const bool typed = inS.type != nullptr && P.nmat > 1;
    const bool attract = has_attraction(P);
    const unsigned b = blocks_for(n, kCollideThreads);
#define DEM_STEP(T, A)                                                                      \
    step_kernel<T, A><<<b, kCollideThreads, 0, st>>>(P, in, inS, cellStart, cellEnd, out,    \
                                                     nextHash, pressure, acc, alpha, errFlag, \
                                                     n)
    if (typed) {
        if (attract) DEM_STEP(true, true); else DEM_STEP(true, false);
    } else {
        if (attract) DEM_STEP(false, true); else DEM_STEP(false, false);
    }
#undef DEM_STEP
    return cudaGetLastError();
}

}  // namespace dem
