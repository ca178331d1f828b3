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

// calcHashD for the batched form: each slot hashes with its specimen's grid.
__global__ void __launch_bounds__(kThreads)
calc_hash_batched_kernel(const KParams* __restrict__ table, const uint32_t* __restrict__ spec,
                         const float2* __restrict__ pos, uint32_t* __restrict__ hash, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const KParams& P = table[spec[i]];
    const int2 g = grid_pos(P, pos[i]);
    hash[i] = grid_hash(P, g.x, g.y);
}

// particles_kernel.cuh:156-233.  A cell starts where the sorted hash differs
// from its predecessor; the predecessor's cell ends there.  The reference
// stages hashes in shared memory; here the neighbour comes from the next lane
// by shuffle and only lane 0 reads hash[i-1] (an L1 hit).
template <bool TYPED>
__global__ void __launch_bounds__(kThreads)
reorder_kernel(uint32_t* __restrict__ cellStart, uint32_t* __restrict__ cellEnd, DynSet s,
               StatSet sS, uint32_t* __restrict__ sLoc, const uint32_t* __restrict__ hash,
               const uint32_t* __restrict__ index, DynSet o, StatSet oS, uint32_t n,
               uint32_t numCells) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    const uint32_t h = valid ? hash[i] : 0u;
    uint32_t hp = __shfl_up_sync(0xffffffffu, h, 1);
    if ((threadIdx.x & 31) == 0 && valid && i > 0) hp = hash[i - 1];
    if (!valid) return;
    // keys outside the grid or indices outside the arrays can only come from a
    // caller's own buffers; such entries are skipped rather than written
    if (i == 0 || h != hp) {
        if (h < numCells) cellStart[h] = i;
        if (i > 0 && hp < numCells) cellEnd[hp] = i;
    }
    if (i == n - 1 && h < numCells) cellEnd[h] = i + 1;
    const uint32_t src = index[i];
    if (src >= n) return;
    s.pos[i] = o.pos[src];
    s.vel[i] = o.vel[src];
    s.theta[i] = o.theta[src];
    s.omega[i] = o.omega[src];
    sS.radius[i] = oS.radius[src];
    sS.mass[i] = oS.mass[src];
    const uint32_t id = oS.id[src];
    sS.id[i] = id;
    if (id < n) sLoc[id] = i;
    if (TYPED) sS.type[i] = oS.type[src];
}

// Cell ranges, read either from the reference's two arrays (cellStart with
// 0xFFFFFFFF for empty cells, cellEnd) or from the context's interleaved
// (start, end) pairs.  An empty cell yields start >= end, so its particle
// loop runs zero times, as the reference's `startIndex != -1` test does.
struct SplitCells {
    const uint32_t* __restrict__ start;
    const uint32_t* __restrict__ end;
    __device__ __forceinline__ uint2 get(uint32_t h) const {
        const uint32_t a = __ldg(start + h);
        return make_uint2(a, a == kEmptyCell ? 0u : __ldg(end + h));
    }
};
struct PackedCells {
    const uint2* __restrict__ range;
    __device__ __forceinline__ uint2 get(uint32_t h) const { return __ldg(range + h); }
};

// Packed pairs of IEEE single-precision operations (PTX f32x2, round to
// nearest even, sm_100): each lane of the result is the same correctly
// rounded value as the scalar operation.
__device__ __forceinline__ float2 f32x2_add(float2 a, float2 b) {
    float2 d;
    asm("{.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 f32x2_sub(float2 a, float2 b) {
    float2 d;
    asm("{.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 f32x2_mul(float2 a, float2 b) {
    float2 d;
    asm("{.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 f32x2_fma(float2 a, float2 b, float2 c) {
    float2 d;
    asm("{.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}

// Contact test and force of one candidate j (the reference's collideSpheres
// and, with ATTRACT, attractSpheres) added to the cell subtotal fc.
template <bool TYPED, bool ATTRACT>
__device__ __forceinline__ void candidate(const KParams& P, uint32_t j, float2 p, float2 v, float w,
                                          float r, uint32_t mat, float2 pj, float d2,
                                          const float2* __restrict__ vel,
                                          const float* __restrict__ omega,
                                          const float* __restrict__ radius,
                                          const uint32_t* __restrict__ type,
                                          const uint32_t* __restrict__ src, float2& fc,
                                          float& moment, float& pr) {
    const float rj = __ldg(radius + j);
    // velocity, spin and type of candidate j sit at its slot of the previous
    // order (src), or at j when the arrays are all in one order (src null)
    const uint32_t sj = src ? __ldg(src + j) : j;
    uint32_t mj = 0;
    float4 pc = P.pair[0];
    if (TYPED) {
        mj = __ldg(type + sj);
        pc = P.pair[mat * P.nmat + mj];
    }
    const float cd = r + rj;
    // d2 > cd^2 (1 + 2e-6) implies sqrtf(d2) >= cd after rounding: no contact
    if (d2 <= cd * cd * 1.000002f && sqrtf(d2) < cd) {
        const float2 f = pair_force(p, pj, v, __ldg(vel + sj), w, __ldg(omega + sj), r, rj, pc,
                                    P.dt, moment, pr);
        fc.x += f.x;
        fc.y += f.y;
    }
    if (ATTRACT) {
        const float2 f = pair_attract(p, pj, r, rj, P.at[mat], P.at[mj], pr);
        fc.x += f.x;
        fc.y += f.y;
    }
}

// Sum of the forces on particle i from its 3x3 cell neighbourhood,
// particles_kernel.cuh:459-549 (collideD) with collideCell (:346-385): cells
// y-outer, x-inner, particles in ascending sorted index, each cell's
// subtotal added to the running force.  `g` is the particle's grid position
// (calcGridPos, or the wrapped cell of its sort key: the same neighbour
// cells).  Wrapping makes a 1- or 2-wide grid visit the same cell more than
// once, exactly as the reference does.
//
// Work the reference spends on pairs that are not in contact is skipped
// without changing any result, because such a pair adds nothing (its force
// is +0 -- and a running sum that starts at +0 can never be -0 -- and it
// touches neither moment nor pressure):
//  * a candidate is dropped before the square root when its squared distance
//    exceeds (rA + rB)^2 by a relative 2e-6; then sqrtf(d2) >= rA + rB after
//    rounding, which is the reference's no-contact branch;
//  * with CULL (the context step, which knows an upper bound rmax on all
//    radii), a neighbour column/row is not visited when the particle is
//    farther than rA + rmax (plus a rounding margin) from that side of its
//    own cell, and candidates are first tested against rA + rmax so that
//    the neighbour's radius is loaded only for near pairs.  Culling needs at
//    least 3 cells per axis and cells wider than 2 rmax (then the three
//    columns/rows are distinct cells and a wrapped neighbour is out of
//    reach) and a particle inside the box by more than the margin.
// `g` is the particle's cell in the context's rows (for a row window, the
// scene's row minus rowOff).
template <bool TYPED, bool ATTRACT, bool CULL, typename Cells>
__device__ __forceinline__ void collide_one(const KParams& P, uint32_t i, int2 g, float2 p,
                                            float2 v, float w, float r, uint32_t mat,
                                            const float2* __restrict__ pos,
                                            const float2* __restrict__ vel,
                                            const float* __restrict__ omega,
                                            const float* __restrict__ radius,
                                            const uint32_t* __restrict__ type,
                                            const uint32_t* __restrict__ src, Cells cells,
                                            float2& force, float& moment, float& pr) {
    force = make_float2(0.0f, 0.0f);
    moment = 0.0f;
    pr = 0.0f;
    int y0 = -1, y1 = 1, x0 = -1, x1 = 1;
    float reach2 = INFINITY;
    if (CULL && p.x > P.cullMargin && p.x < P.Lx - P.cullMargin && p.y > P.cullMargin &&
        p.y < P.Ly - P.cullMargin) {
        const float reach = (r + P.rmax) * 1.0001f + P.cullMargin;
        // the cell's lower corner; a row window's rows are the scene's from rowOff
        const float X0 = (float)g.x * P.cellW, Y0 = (float)(g.y + P.rowOff) * P.cellH;
        if (p.x - X0 > reach) x0 = 0;
        if (X0 + P.cellW - p.x > reach) x1 = 0;
        if (p.y - Y0 > reach) y0 = 0;
        if (Y0 + P.cellH - p.y > reach) y1 = 0;
        const float rr = (r + P.rmax) * 1.0001f;
        reach2 = rr * rr;
    }
#pragma unroll 1
    for (int dy = y0; dy <= y1; ++dy) {
#pragma unroll 1
        for (int dx = x0; dx <= x1; ++dx) {
            const uint2 se = cells.get(cell_index(P, g.x + dx, g.y + dy));
            float2 fc = make_float2(0.0f, 0.0f);
            // empty cells have start >= end (start 0xFFFFFFFF): no iterations
            const uint32_t count = se.y > se.x ? se.y - se.x : 0u;
            const uint32_t stop = se.x + (count & ~1u);
            uint32_t j = se.x;
            // two candidates per iteration: two loads in flight
#pragma unroll 1
            for (; j < stop; j += 2) {
                const float2 pa = __ldg(pos + j);
                const float2 pb = __ldg(pos + j + 1);
                const float ax = pa.x - p.x, ay = pa.y - p.y;
                const float bx = pb.x - p.x, by = pb.y - p.y;
                const float da = ax * ax + ay * ay;
                const float db = bx * bx + by * by;
                if (j != i && (ATTRACT || !CULL || da <= reach2))
                    candidate<TYPED, ATTRACT>(P, j, p, v, w, r, mat, pa, da, vel, omega, radius,
                                              type, src, fc, moment, pr);
                if (j + 1 != i && (ATTRACT || !CULL || db <= reach2))
                    candidate<TYPED, ATTRACT>(P, j + 1, p, v, w, r, mat, pb, db, vel, omega,
                                              radius, type, src, fc, moment, pr);
            }
            if ((count & 1u) && j != i) {
                const float2 pa = __ldg(pos + j);
                const float ax = pa.x - p.x, ay = pa.y - p.y;
                const float da = ax * ax + ay * ay;
                if (ATTRACT || !CULL || da <= reach2)
                    candidate<TYPED, ATTRACT>(P, j, p, v, w, r, mat, pa, da, vel, omega, radius,
                                              type, src, fc, moment, pr);
            }
            force.x += fc.x;
            force.y += fc.y;
        }
    }
}

// Row-interval form of collide_one for the context step (no attraction, no
// x-wrap among the visited columns).  The cells (cx-1, cx, cx+1) of one row
// are consecutive cells, so their particles form one contiguous index
// interval in sorted order, read from the first-particle array (cellFirst).
// A lane walks the interval of each row it visits after culling, one row
// after the other, so the lanes of a warp run about as many iterations as
// their own candidates in that row instead of the per-cell maximum.
// Positions and radii are in sorted order; a contact's velocity, spin and
// type are read at the neighbour's slot of the previous order, src[j].
//
// Each interval is walked twice, in chunks of 32 candidates: a lean filter
// sets one bit per candidate whose squared distance is within
// (rA + rB)^2 (1 + 2e-6), up to rounding -- a superset of the contacts -- and the contact
// law then runs on the set bits in increasing index.  The law's own
// `dist < rA + rB` test rejects the few non-contacts among them with a +0
// force, which changes no sum, so every contact is met in the same
// (row, index) order as before.  Keeping the law out of the filter loop
// means a warp runs it once per contact of its busiest lane rather than once
// per candidate slot in which any lane has a contact.
//
// The summation order is the reference's: the cell a contact belongs to is
// found from the cell boundaries, each row keeps one subtotal per cell and
// adds them to the force in cell order at the end of the row (an empty or
// culled cell adds +0, which changes nothing).  Returns false, without
// touching the outputs, when the visited columns wrap; the caller then uses
// collide_one.
template <bool TYPED>
__device__ __forceinline__ bool collide_rows(const KParams& P, uint32_t i, int2 g, float2 p,
                                             float2 v, float w, float r, uint32_t mat,
                                             const float2* __restrict__ pos,
                                             const float2* __restrict__ vel,
                                             const float* __restrict__ omega,
                                             const float* __restrict__ radius,
                                             const uint32_t* __restrict__ type,
                                             const uint32_t* __restrict__ src,
                                             const uint32_t* __restrict__ cellFirst,
                                             float2& force, float& moment, float& pr) {
    int y0 = -1, y1 = 1, x0 = -1, x1 = 1;
    if (p.x > P.cullMargin && p.x < P.Lx - P.cullMargin && p.y > P.cullMargin &&
        p.y < P.Ly - P.cullMargin) {
        const float reach = (r + P.rmax) * 1.0001f + P.cullMargin;
        const float X0 = (float)g.x * P.cellW, Y0 = (float)(g.y + P.rowOff) * P.cellH;
        if (p.x - X0 > reach) x0 = 0;
        if (X0 + P.cellW - p.x > reach) x1 = 0;
        if (p.y - Y0 > reach) y0 = 0;
        if (Y0 + P.cellH - p.y > reach) y1 = 0;
    }
    if (g.x + x0 < 0 || g.x + x1 >= (int)P.gx) return false;
    force = make_float2(0.0f, 0.0f);
    moment = 0.0f;
    pr = 0.0f;
    const float4 pc0 = P.pair[0];
#pragma unroll 1
    for (int dy = y0; dy <= y1; ++dy) {
        const uint32_t row = P.cellOff + (uint32_t)((g.y + dy) & (int)(P.gy - 1u)) * P.gx;
        // the visited cells of this row are first = x0 .. x1; visited cell k
        // holds the particles
        // [start[first + k], start[first + k + 1]); a contact at index j
        // belongs to visited cell (j >= b1) + (j >= b2)
        const uint32_t* __restrict__ sc = cellFirst + (row + (uint32_t)(g.x + x0));
        const uint32_t o0 = __ldg(sc), o1 = __ldg(sc + 1), o2 = __ldg(sc + 2), o3 = __ldg(sc + 3);
        const int span = x1 - x0;  // visited cells - 1
        const uint32_t a = o0;
        const uint32_t b = span == 0 ? o1 : (span == 1 ? o2 : o3);
        const uint32_t b1 = span >= 1 ? o1 : 0xffffffffu;
        const uint32_t b2 = span >= 2 ? o2 : 0xffffffffu;
        float2 f0 = make_float2(0.0f, 0.0f), f1 = f0, f2 = f0;
        // filter: a bit per candidate that may touch, then the contact law on
        // the set bits in index order.  Groups of 8 candidates are read whole
        // (the arrays are padded by kFilterPad), the bits past the interval
        // and the particle's own bit are cleared per chunk.  Two candidates
        // share each packed f32x2 operation.  d2 is the law's own
        // rn(rn(dx^2) + rn(dy^2)); the bound cd^2 (1 + 2e-6) is a fused
        // multiply-add, within 2e-7 relative of the exact value, so a
        // rejected candidate still has sqrtf(d2) >= rA + rB in the law's
        // arithmetic (the law itself is unchanged).
#pragma unroll 1
        for (uint32_t base = a; base < b; base += 32u) {
            const uint32_t cnt = min(b - base, 32u);
            uint32_t mask = 0u;
#pragma unroll 1
            for (uint32_t k0 = 0; k0 < cnt; k0 += 8) {
                float2 q[8];
                float rq[8];
                const float2* __restrict__ pq = pos + (base + k0);
                const float* __restrict__ pr8 = radius + (base + k0);
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    q[k] = __ldg(pq + k);
                    rq[k] = __ldg(pr8 + k);
                }
                uint32_t m8 = 0u;
#pragma unroll
                for (int k = 0; k < 8; k += 2) {
                    const float2 da = f32x2_sub(q[k], p), db = f32x2_sub(q[k + 1], p);
                    const float2 sa = f32x2_mul(da, da), sb = f32x2_mul(db, db);
                    const float d2a = sa.x + sa.y, d2b = sb.x + sb.y;
                    const float2 cd = f32x2_add(make_float2(r, r), make_float2(rq[k], rq[k + 1]));
                    const float2 c2 = f32x2_mul(cd, cd);
                    const float2 bound = f32x2_fma(c2, make_float2(2e-6f, 2e-6f), c2);
                    if (d2a <= bound.x) m8 |= 1u << k;
                    if (d2b <= bound.y) m8 |= 2u << k;
                }
                mask |= m8 << k0;
            }
            if (cnt < 32u) mask &= (1u << cnt) - 1u;
            if (i - base < 32u) mask &= ~(1u << (i - base));
            while (mask) {
                const uint32_t j = base + (uint32_t)(__ffs(mask) - 1);
                mask &= mask - 1u;
                const float rj = __ldg(radius + j);
                float4 pc = pc0;
                const uint32_t sj = __ldg(src + j);
                if (TYPED) pc = P.pair[mat * P.nmat + __ldg(type + sj)];
                const float2 f = pair_force(p, __ldg(pos + j), v, __ldg(vel + sj), w, __ldg(omega + sj),
                                            r, rj, pc, P.dt, moment, pr);
                if (j >= b2) { f2.x += f.x; f2.y += f.y; }
                else if (j >= b1) { f1.x += f.x; f1.y += f.y; }
                else { f0.x += f.x; f0.y += f.y; }
            }
        }
        force.x += f0.x; force.y += f0.y;
        force.x += f1.x; force.y += f1.y;
        force.x += f2.x; force.y += f2.y;
    }
    return true;
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
    int2 g = grid_pos(P, p);
    g.y -= P.rowOff;  // collide_one takes the cell in the context's rows
    collide_one<TYPED, ATTRACT, false>(P, i, g, p, v, w, r, mat, pos, vel, omega,
                                       radius, type, nullptr, SplitCells{cellStart, cellEnd}, f,
                                       moment, pr);
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

// collide_one/rows/staged done: acceleration, integration, next hash, mover
// record (shared tail of step_kernel).  `m` and `s.th` were read with the
// particle's other fields before the collide, so no load waits here.
template <bool TYPED>
__device__ __forceinline__ void finish_particle(
    const KParams& P, uint32_t i, Dyn& s, float2 f, float moment, float pr, float r, float m,
    uint32_t mat, uint32_t id, uint32_t key, const uint2* __restrict__ cellRange, DynSet out,
    StatSet outS, uint32_t* __restrict__ loc, uint32_t* __restrict__ nextHash,
    float* __restrict__ pressure, float2* __restrict__ acc, float* __restrict__ alpha,
    uint32_t* __restrict__ errFlag, MoverSinkArgs sink) {
    // F/m and M/I as the reference divides them.  Without contacts F and M
    // are +0 (sums that start at +0 never become -0), and +0 divided by a
    // positive finite mass or inertia is exactly +0, so the divisions are
    // skipped then; 2 m r^2 in [1e-30, 1e30] keeps the inertia positive and
    // finite.
    const bool quiet = f.x == 0.0f && f.y == 0.0f && moment == 0.0f && m > 0.0f && m < INFINITY;
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
    if (acc) acc[i] = a;
    if (alpha) alpha[i] = al;
    integrate_one(P, s, a, al, r, m, mat, pr);
    // the new state in this step's sorted order
    out.pos[i] = s.p;
    out.vel[i] = s.v;
    out.theta[i] = s.th;
    out.omega[i] = s.w;
    outS.mass[i] = m;
    outS.id[i] = id;
    if (TYPED) outS.type[i] = mat;
    loc[id] = i;
    if (pressure) pressure[i] = pr;
    const int2 gn = grid_pos_fast(P, s.p);
    const uint32_t nk = grid_hash(P, gn.x, gn.y);
    nextHash[i] = nk;
    if (!(isfinite(s.p.x) && isfinite(s.p.y))) atomicOr(errFlag, 1u);
    if (sink.ctrl && nk != key) {
        // a mover: count it as a leaver of its cell and an arrival of the new
        // one, and record it for the next step's incremental sort
        const uint32_t slot = atomicAdd(sink.arrCnt + nk, 1u);
        atomicAdd(sink.leavers + key, 1u);
        if (nk > key) atomicAdd(sink.arrLo + nk, 1u);
        const uint32_t m = atomicAdd(sink.ctrl + 1, 1u);
        const uint2 own = cellRange[key];
        if (m < sink.moverCap) sink.movers[m] = make_uint4(i, nk, key, slot);
        if (m >= sink.moverCap || slot >= kMaxGroup || own.y - own.x > kMaxGroup)
            atomicOr(sink.ctrl, 1u);
        // the cell scan rescans the tiles of both cells
        if (sink.dirty) {
            const uint32_t t0 = key >> sink.tileShift, t1 = nk >> sink.tileShift;
            atomicOr(sink.dirty + (t0 >> 5), 1u << (t0 & 31u));
            if (t1 != t0) atomicOr(sink.dirty + (t1 >> 5), 1u << (t1 & 31u));
        }
    }
}

// collideD + integrateSystemD + calcHashD of the next step for one particle.
// The acceleration stays in registers instead of a round trip through HBM;
// the arithmetic is the same expressions in the same order.
template <bool TYPED, bool ATTRACT, bool CULL, bool CONTROL = false>
__device__ __forceinline__ void step_particle(const KParams& P, uint32_t i, DynSet in,
                                              StatSet inS, const uint32_t* __restrict__ src,
                                              const uint32_t* __restrict__ sortedKey,
                                              const uint2* __restrict__ cellRange,
                                              const uint32_t* __restrict__ cellFirst, DynSet out,
                                              StatSet outS, uint32_t* __restrict__ loc,
                                              uint32_t* __restrict__ nextHash,
                                              float* __restrict__ pressure,
                                              float2* __restrict__ acc,
                                              float* __restrict__ alpha,
                                              uint32_t* __restrict__ errFlag, MoverSinkArgs sink,
                                              ControlArgs ctl = ControlArgs{}) {
    // position and radius are in this step's sorted order; the other fields
    // at the particle's slot of the previous order, src[i]
    Dyn s;
    s.p = in.pos[i];
    const float r = inS.radius[i];
    const uint32_t si = src[i];
    s.v = in.vel[si];
    s.w = in.omega[si];
    s.th = in.theta[si];
    const float m = inS.mass[si];
    const uint32_t id = inS.id[si];
    const uint32_t mat = TYPED ? inS.type[si] : 0u;
    // the sort key of particle i is calcGridPos of this very position, wrapped
    const uint32_t key = sortedKey[i];
    const uint32_t local = key - P.cellOff;
    const int2 g = make_int2((int)(local & (P.gx - 1u)), (int)(local >> P.log2gx));
    float2 f;
    float moment, pr;
    if (ATTRACT || !CULL || !P.cull ||
        !collide_rows<TYPED>(P, i, g, s.p, s.v, s.w, r, mat, in.pos, in.vel, in.omega,
                             inS.radius, inS.type, src, cellFirst, f, moment, pr)) {
        if (CULL && P.cull)
            collide_one<TYPED, ATTRACT, true>(P, i, g, s.p, s.v, s.w, r, mat, in.pos, in.vel,
                                              in.omega, inS.radius, inS.type, src,
                                              PackedCells{cellRange}, f, moment, pr);
        else
            collide_one<TYPED, ATTRACT, false>(P, i, g, s.p, s.v, s.w, r, mat, in.pos, in.vel,
                                               in.omega, inS.radius, inS.type, src,
                                               PackedCells{cellRange}, f, moment, pr);
    }
    if (CONTROL) {
        // particles_kernel.cuh:520-541: the contact (and attraction) with the
        // control particle after the 3x3 cells; its force is added once, the
        // reaction is stored for the reduction
        const ControlDev c = *ctl.c;
        const float4 pc = TYPED ? P.pair[mat * P.nmat + c.mat] : P.pair[0];
        float mc = 0.0f;
        float2 fc = pair_force(s.p, c.pos, s.v, c.vel, s.w, c.omega, r, c.radius, pc, P.dt, mc,
                               pr);
        if (ATTRACT) {
            const float2 fa = pair_attract(s.p, c.pos, r, c.radius, P.at[mat], P.at[c.mat], pr);
            fc.x += fa.x;
            fc.y += fa.y;
        }
        f.x += fc.x;
        f.y += fc.y;
        moment += mc;
        ctl.fx[i] = -fc.x;
        ctl.fy[i] = -fc.y;
        ctl.fm[i] = -mc / r * c.radius;
    }
    finish_particle<TYPED>(P, i, s, f, moment, pr, r, m, mat, id, key, cellRange, out, outS, loc,
                           nextHash, pressure, acc, alpha, errFlag, sink);
}

// THREADS x MINB: the block size and the blocks per SM the registers are
// capped for (the step variants, chosen by the context's autotuner).
template <bool TYPED, bool ATTRACT, bool CULL, bool CONTROL, int THREADS = kCollideThreads,
          int MINB = 1024 / kCollideThreads>
__global__ void __launch_bounds__(THREADS, MINB)
step_kernel(KParams P, DynSet in, StatSet inS, const uint32_t* __restrict__ src,
            const uint32_t* __restrict__ sortedKey, const uint2* __restrict__ cellRange,
            const uint32_t* __restrict__ cellFirst, DynSet out, StatSet outS,
            uint32_t* __restrict__ loc, uint32_t* __restrict__ nextHash,
            float* __restrict__ pressure, float2* __restrict__ acc, float* __restrict__ alpha,
            uint32_t* __restrict__ errFlag, uint32_t n, MoverSinkArgs sink, ControlArgs ctl) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    step_particle<TYPED, ATTRACT, CULL, CONTROL>(P, i, in, inS, src, sortedKey, cellRange,
                                                 cellFirst, out, outS, loc, nextHash, pressure,
                                                 acc, alpha, errFlag, sink, ctl);
}

// reduceVecD (particles_kernel.cuh:551-578) for the three reaction vectors,
// launched as collide launches it (functions.cu:486-488): blocks of
// min(512, n) threads, a shared-memory tree that halves the block size.
constexpr int kControlThreads = 512;
__global__ void __launch_bounds__(kControlThreads)
control_reduce_kernel(ControlArgs ctl, uint32_t n, float* __restrict__ partials) {
    __shared__ float cache[3][kControlThreads];
    const uint32_t index = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = threadIdx.x;
    const bool in = index < n;
    cache[0][t] = in ? ctl.fx[index] : 0.0f;
    cache[1][t] = in ? ctl.fy[index] : 0.0f;
    cache[2][t] = in ? ctl.fm[index] : 0.0f;
    __syncthreads();
    for (int i = blockDim.x / 2; i != 0; i /= 2) {
        if (t < i) {
            cache[0][t] += cache[0][t + i];
            cache[1][t] += cache[1][t + i];
            cache[2][t] += cache[2][t + i];
        }
        __syncthreads();
    }
    if (t == 0) {
        partials[blockIdx.x] = cache[0][0];
        partials[gridDim.x + blockIdx.x] = cache[1][0];
        partials[2 * gridDim.x + blockIdx.x] = cache[2][0];
    }
}

// the host's sum of the block results in block order (functions.cu:511-519),
// then the host's move of the control particle (main.cu:511-514): float +=
// double, and the wraps
__global__ void control_sum_move_kernel(ControlDev* __restrict__ c,
                                        const float* __restrict__ partials, uint32_t blocks,
                                        float* __restrict__ out) {
    float sx = 0.0f, sy = 0.0f, sm = 0.0f;
    for (uint32_t b = 0; b < blocks; ++b) {
        sx += partials[b];
        sy += partials[blocks + b];
        sm += partials[2 * blocks + b];
    }
    out[0] = sx;
    out[1] = sy;
    out[2] = sm;
    float2 p = c->pos;
    p.x = (float)((double)p.x + c->drift[0]);
    p.y = (float)((double)p.y + c->drift[1]);
    if ((double)p.y < c->wrapYBelow) p.y = (float)c->wrapYTo;
    if ((double)p.x > c->wrapXAbove) p.x = (float)c->wrapXTo;
    c->pos = p;
}

// Batched form: particle slot i belongs to specimen spec[i] (slots of a
// specimen are contiguous and never change specimen), whose parameters --
// box, grid, cell offset, contact coefficients -- come from a device table.
template <bool TYPED, bool ATTRACT, bool CULL, int THREADS = kCollideThreads,
          int MINB = 1024 / kCollideThreads>
__global__ void __launch_bounds__(THREADS, MINB)
step_kernel_batched(const KParams* __restrict__ table, const uint32_t* __restrict__ spec,
                    DynSet in, StatSet inS, const uint32_t* __restrict__ src,
                    const uint32_t* __restrict__ sortedKey, const uint2* __restrict__ cellRange,
                    const uint32_t* __restrict__ cellFirst, DynSet out, StatSet outS,
                    uint32_t* __restrict__ loc, uint32_t* __restrict__ nextHash,
                    float* __restrict__ pressure, float2* __restrict__ acc,
                    float* __restrict__ alpha, uint32_t* __restrict__ errFlag, uint32_t n,
                    MoverSinkArgs sink) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    step_particle<TYPED, ATTRACT, CULL>(table[spec[i]], i, in, inS, src, sortedKey, cellRange,
                                        cellFirst, out, outS, loc, nextHash, pressure, acc,
                                        alpha, errFlag, sink);
}

// Reorder for the context step: as reorder_kernel, but the cell ranges are
// written as interleaved (start, end) pairs (empty cells hold 0xFFFFFFFF).
template <bool TYPED>
__global__ void __launch_bounds__(kThreads)
reorder_packed_kernel(uint2* __restrict__ cellRange, DynSet s, StatSet sS,
                      uint32_t* __restrict__ sLoc, const uint32_t* __restrict__ hash,
                      const uint32_t* __restrict__ index, DynSet o, StatSet oS, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    const uint32_t h = valid ? hash[i] : 0u;
    uint32_t hp = __shfl_up_sync(0xffffffffu, h, 1);
    if ((threadIdx.x & 31) == 0 && valid && i > 0) hp = hash[i - 1];
    if (!valid) return;
    if (i == 0 || h != hp) {
        cellRange[h].x = i;
        if (i > 0) cellRange[hp].y = i;
    }
    if (i == n - 1) cellRange[h].y = i + 1;
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

__global__ void unpack_cells_kernel(const uint2* __restrict__ range, uint32_t numCells,
                                    uint32_t* __restrict__ cellStart,
                                    uint32_t* __restrict__ cellEnd) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= numCells) return;
    const uint2 v = range[c];
    if (cellStart) cellStart[c] = v.x;
    if (cellEnd) cellEnd[c] = v.y;
}

// One row of the reference's followed-particle output (functions.cu:630-654)
// for the particle in slot i: id, type, pos, vel, acc, theta, omega, alpha,
// pressure.
__device__ __forceinline__ void followed_row(uint32_t i, float* __restrict__ r, const DynSet& d,
                                             const StatSet& s, const float2* __restrict__ acc,
                                             const float* __restrict__ alpha,
                                             const float* __restrict__ pressure) {
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

__global__ void followed_kernel(FollowIds f, const uint32_t* __restrict__ loc, DynSet d, StatSet s,
                                const float2* __restrict__ acc, const float* __restrict__ alpha,
                                const float* __restrict__ pressure, float* __restrict__ rows) {
    const uint32_t k = threadIdx.x;
    if (k >= f.count) return;
    followed_row(loc[f.id[k]], rows + 12 * k, d, s, acc, alpha, pressure);
}

// The rows of ids[0, *count) into row block (slot ? *slot : 0) + add of
// `ring` (*count rows of 12 words per block).
__global__ void followed_ring_kernel(const uint32_t* __restrict__ ids,
                                     const uint32_t* __restrict__ countWord,
                                     const uint32_t* __restrict__ slot, uint32_t add,
                                     const uint32_t* __restrict__ loc, DynSet d, StatSet s,
                                     const float2* __restrict__ acc,
                                     const float* __restrict__ alpha,
                                     const float* __restrict__ pressure, float* __restrict__ ring) {
    const uint32_t count = *countWord;
    float* base = ring + (size_t)((slot ? *slot : 0u) + add) * count * 12;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x)
        followed_row(loc[ids[k]], base + 12ull * k, d, s, acc, alpha, pressure);
}

// Largest radius (positive floats order like their bit patterns).
__global__ void max_radius_kernel(const float* __restrict__ radius, uint32_t n,
                                  uint32_t* __restrict__ out) {
    float m = 0.0f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        m = fmaxf(m, radius[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
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

cudaError_t launch_followed_ring(const uint32_t* ids, const uint32_t* countWord,
                                 const uint32_t* slot, uint32_t add, const uint32_t* loc, DynSet d,
                                 StatSet s, const float2* acc, const float* alpha,
                                 const float* pressure, float* ring, cudaStream_t st) {
    followed_ring_kernel<<<16, 128, 0, st>>>(ids, countWord, slot, add, loc, d, s, acc, alpha,
                                             pressure, ring);
    return cudaGetLastError();
}

cudaError_t launch_max_radius(const float* radius, uint32_t n, uint32_t* out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess || n == 0) return e;
    const unsigned b = blocks_for(n, kThreads) < 1184 ? blocks_for(n, kThreads) : 1184;
    max_radius_kernel<<<b, kThreads, 0, st>>>(radius, n, out);
    return cudaGetLastError();
}

cudaError_t launch_calc_hash_batched(const KParams* table, const uint32_t* spec, const float2* pos,
                                     uint32_t* hash, uint32_t n, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    calc_hash_batched_kernel<<<blocks_for(n, kThreads), kThreads, 0, st>>>(table, spec, pos, hash,
                                                                           n);
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
            cellStart, cellEnd, sorted, sortedS, sortedLoc, hash, index, old, oldS, n, numCells);
    else
        reorder_kernel<false><<<blocks_for(n, kThreads), kThreads, 0, st>>>(
            cellStart, cellEnd, sorted, sortedS, sortedLoc, hash, index, old, oldS, n, numCells);
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

cudaError_t launch_step(const KParams& P, DynSet in, StatSet inS, const uint32_t* src,
                        const uint32_t* sortedKey, const uint2* cellRange,
                        const uint32_t* cellFirst, DynSet out, StatSet outS, uint32_t* loc,
                        uint32_t* nextHash, float* pressure, float2* acc, float* alpha,
                        uint32_t* errFlag, uint32_t n, MoverSinkArgs sink, cudaStream_t st,
                        const KParams* table, const uint32_t* spec, ControlArgs ctl,
                        int variant) {
    if (n == 0) return cudaSuccess;
    if (variant < 0 || variant >= kStepVariants) return cudaErrorInvalidValue;
    const bool typed = inS.type != nullptr && P.nmat > 1;
    const bool attract = has_attraction(P);
    const bool cull = table ? true : P.cull != 0u;
#define DEM_STEP_T(T, A, C, TH, MB)                                                            \
    do {                                                                                       \
        const unsigned b = blocks_for(n, TH);                                                  \
        if (table)                                                                             \
            step_kernel_batched<T, A, C, TH, MB><<<b, TH, 0, st>>>(                            \
                table, spec, in, inS, src, sortedKey, cellRange, cellFirst, out, outS, loc,     \
                nextHash, pressure, acc, alpha, \
                errFlag, n, sink);                                                             \
        else if (ctl.c)                                                                        \
            step_kernel<T, A, C, true><<<blocks_for(n, kCollideThreads), kCollideThreads, 0,  \
                                         st>>>(P, in, inS, src, sortedKey, cellRange, cellFirst, \
                                               out, outS, loc, nextHash, \
                                               pressure, acc, alpha, errFlag, n, sink, ctl);  \
        else                                                                                   \
            step_kernel<T, A, C, false, TH, MB><<<b, TH, 0, st>>>(                             \
                P, in, inS, src, sortedKey, cellRange, cellFirst, out, outS, loc, nextHash,    \
                pressure, acc, alpha, errFlag, \
                n, sink, ctl);                                                                 \
    } while (0)
#define DEM_STEP(T, A, C)                                                                      \
    do {                                                                                       \
        switch (variant) {                                                                     \
            case 1: DEM_STEP_T(T, A, C, 64, 16); break;                                        \
            case 2: DEM_STEP_T(T, A, C, 256, 4); break;                                        \
            case 3: DEM_STEP_T(T, A, C, 128, 6); break;                                        \
            default: DEM_STEP_T(T, A, C, 128, 8); break;                                       \
        }                                                                                      \
    } while (0)
    if (typed) {
        if (attract) DEM_STEP(true, true, false);
        else if (cull) DEM_STEP(true, false, true);
        else DEM_STEP(true, false, false);
    } else {
        if (attract) DEM_STEP(false, true, false);
        else if (cull) DEM_STEP(false, false, true);
        else DEM_STEP(false, false, false);
    }
#undef DEM_STEP
#undef DEM_STEP_T
    return cudaGetLastError();
}

StepShape step_variant_shape(int variant) {
    switch (variant) {
        case 1: return StepShape{64, 16};
        case 2: return StepShape{256, 4};
        case 3: return StepShape{128, 6};
        default: return StepShape{128, 8};
    }
}

namespace {
__global__ void loop_init_kernel(const uint32_t* __restrict__ req, uint32_t* __restrict__ left,
                                 cudaGraphConditionalHandle h) {
    const uint32_t n = *req;
    *left = n;
    cudaGraphSetConditional(h, n ? 1u : 0u);
}
__global__ void loop_next_kernel(uint32_t* __restrict__ left, uint32_t* __restrict__ idx,
                                 int32_t idxStep, cudaGraphConditionalHandle h) {
    const uint32_t n = *left - 1u;
    *left = n;
    if (idx) *idx += (uint32_t)idxStep;
    cudaGraphSetConditional(h, n ? 1u : 0u);
}
}  // namespace

namespace {
__global__ void set_words_kernel(uint32_t* __restrict__ dst, Words w) {
    for (uint32_t i = 0; i < w.count; ++i) dst[i] = w.v[i];
}
}  // namespace

cudaError_t launch_set_words(uint32_t* dst, Words w, cudaStream_t st) {
    if (w.count > 8) return cudaErrorInvalidValue;
    set_words_kernel<<<1, 1, 0, st>>>(dst, w);
    return cudaGetLastError();
}

cudaError_t launch_loop_init(const uint32_t* req, uint32_t* left, cudaGraphConditionalHandle h,
                             cudaStream_t st) {
    loop_init_kernel<<<1, 1, 0, st>>>(req, left, h);
    return cudaGetLastError();
}

cudaError_t launch_loop_next(uint32_t* left, uint32_t* idx, int32_t idxStep,
                             cudaGraphConditionalHandle h, cudaStream_t st) {
    loop_next_kernel<<<1, 1, 0, st>>>(left, idx, idxStep, h);
    return cudaGetLastError();
}

cudaError_t launch_control_post(ControlArgs ctl, ControlDev* c, uint32_t n, float* partials,
                                float* out, cudaStream_t st, int* launches) {
    const uint32_t threads = n < (uint32_t)kControlThreads ? (n ? n : 1u) : (uint32_t)kControlThreads;
    const uint32_t blocks = n ? (n + threads - 1) / threads : 0u;
    if (blocks) control_reduce_kernel<<<blocks, threads, 0, st>>>(ctl, n, partials);
    control_sum_move_kernel<<<1, 1, 0, st>>>(c, partials, blocks, out);
    if (launches) *launches += blocks ? 2 : 1;
    return cudaGetLastError();
}

cudaError_t launch_reorder_packed(uint2* cellRange, DynSet sorted, StatSet sortedS,
                                  uint32_t* sortedLoc, const uint32_t* hash, const uint32_t* index,
                                  DynSet old, StatSet oldS, uint32_t n, uint32_t numCells,
                                  cudaStream_t st, int* launches) {
    cudaError_t e = cudaMemsetAsync(cellRange, 0xff, sizeof(uint2) * (size_t)numCells, st);
    if (e != cudaSuccess || n == 0) return e;
    if (sortedS.type && oldS.type)
        reorder_packed_kernel<true><<<blocks_for(n, kThreads), kThreads, 0, st>>>(
            cellRange, sorted, sortedS, sortedLoc, hash, index, old, oldS, n);
    else
        reorder_packed_kernel<false><<<blocks_for(n, kThreads), kThreads, 0, st>>>(
            cellRange, sorted, sortedS, sortedLoc, hash, index, old, oldS, n);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t launch_unpack_cells(const uint2* cellRange, uint32_t numCells, uint32_t* cellStart,
                                uint32_t* cellEnd, cudaStream_t st) {
    if (numCells == 0) return cudaSuccess;
    unpack_cells_kernel<<<blocks_for(numCells, kThreads), kThreads, 0, st>>>(cellRange, numCells,
                                                                             cellStart, cellEnd);
    return cudaGetLastError();
}

}  // namespace dem
