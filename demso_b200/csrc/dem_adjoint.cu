// Adjoint of the DEM step: reverse-mode gradients of a scalar loss with
// respect to the initial state and the contact coefficients.
//
// Forward: dem_adj_forward steps the context as dem_step does and keeps a
// checkpoint of the state every `every` steps.  Backward: for each window,
// last first, the checkpoint is restored and the window re-run while
// recording, per step, the sorted state, the cell ranges and the
// accelerations; then the window's steps are reversed:
//   integrate VJP (per particle): walls, floor contact and the symplectic
//     Euler update, giving the cotangents of the contact force F and moment M;
//   pair VJP (per particle, gather over the same 3x3 cells as collide): for
//     a contact (i, j) the force on j is exactly minus the force on i and the
//     moment term Ft.t is the same from both sides, so particle i needs only
//     (lamF_i - lamF_j) and (lamM_i r_i + lamM_j r_j) -- no atomics; the
//     Jacobian of the contact law comes from forward-mode duals evaluated on
//     the recorded float values, so every branch (contact, dashpot, stick or
//     slip, walls) is the one the forward took ("frozen contact set");
//   coefficient gradients are summed in double: per warp over the slots of
//     one specimen, into per-slot accumulators, then per specimen in a fixed
//     order, so they are deterministic.
// A batch (dem_batch_create) is differentiated the same way, each slot
// reading its specimen's parameters; the coefficient gradients come out per
// specimen.
// The state adjoints live in particle-id order between steps.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/demso_b200.h"
#include "dem_common.cuh"
#include "dem_dual.cuh"
#include "dem_kernels.cuh"

namespace dem {
namespace {

constexpr int kAdjThreads = 128;
constexpr int kCoef = DEM_ADJ_NUM_COEF;  // kn, kt, cn, mu (pairs), cn, mu, kt (floor)

inline unsigned blocks_for(uint32_t n, int t) { return (n + (uint32_t)t - 1u) / (uint32_t)t; }
inline size_t al256(size_t b) { return (b + 255u) & ~(size_t)255u; }

// One recorded step: the sorted state the step kernel read, its cell ranges
// and the accelerations it computed.
struct StepRec {
    float2* pos;
    float2* vel;
    float* omega;
    float* radius;
    float* mass;
    uint32_t* id;
    float2* acc;
    float* alpha;
    uint2* cells;
};

template <typename T>
__device__ __forceinline__ T* bump(T* p, size_t off) {
    return reinterpret_cast<T*>(reinterpret_cast<char*>(p) + off);
}
// The record `at` names (see RecSlot), from the one at the window's base.
__device__ __forceinline__ StepRec rec_at(StepRec r, RecSlot at) {
    if (!at.slot) return r;
    const size_t off = at.stride * (size_t)(*at.slot + at.add);
    r.pos = bump(r.pos, off);
    r.vel = bump(r.vel, off);
    r.omega = bump(r.omega, off);
    r.radius = bump(r.radius, off);
    r.mass = bump(r.mass, off);
    r.id = bump(r.id, off);
    r.acc = bump(r.acc, off);
    r.alpha = bump(r.alpha, off);
    r.cells = bump(r.cells, off);
    return r;
}

// Adds a thread's coefficient cotangents to the per-slot accumulators
// acc[k * n + slot]: the values of a warp are reduced over runs of equal
// `seg` (slots of one specimen are contiguous) in a fixed pattern, and the
// first lane of each run adds the run's sum to its own slot.  Every slot is
// always summed by the same lanes in the same order, so the result does not
// depend on scheduling.
__device__ __forceinline__ void warp_add_coef(const double (&v)[kCoef], uint32_t seg, uint32_t i,
                                              uint32_t n, double* __restrict__ acc) {
    const int lane = threadIdx.x & 31;
    const uint32_t prev = __shfl_up_sync(0xffffffffu, seg, 1);
    const bool head = i < n && (lane == 0 || prev != seg);
#pragma unroll
    for (int k = 0; k < kCoef; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double y = __shfl_down_sync(0xffffffffu, x, o);
            const uint32_t so = __shfl_down_sync(0xffffffffu, seg, o);
            if (lane + o < 32 && so == seg) x += y;
        }
        if (head && x != 0.0) acc[(size_t)k * n + i] += x;
    }
}

// Reverse of integrate_one (particles_kernel.cuh:580-627) for one particle.
__global__ void __launch_bounds__(kAdjThreads)
adj_integrate_kernel(KParams P0, const KParams* __restrict__ table,
                     const uint32_t* __restrict__ spec, StepRec rec0, RecSlot at, uint32_t n,
                     const float2* __restrict__ lamXin, const float2* __restrict__ lamVin,
                     const float* __restrict__ lamWin, float2* __restrict__ lx,
                     float2* __restrict__ lv, float* __restrict__ lw, float2* __restrict__ lamF,
                     float* __restrict__ lamM, double* __restrict__ acc) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double coef[kCoef] = {0, 0, 0, 0, 0, 0, 0};
    const uint32_t seg = i < n ? (table ? spec[i] : 0u) : 0xffffffffu;
    if (i < n) {
        const StepRec rec = rec_at(rec0, at);
        const KParams& P = table ? table[seg] : P0;
        const uint32_t id = rec.id[i];
        const float r = rec.radius[i], m = rec.mass[i];
        const float I = inertia_of(m, r);
        const float2 x = rec.pos[i], v = rec.vel[i], a = rec.acc[i];
        const float w = rec.omega[i], al = rec.alpha[i];
        const float eb = P.eb[0];
        // forward, keeping what the reverse needs
        float2 v1 = make_float2(v.x + (P.gravx + a.x) * P.dt, v.y + (P.gravy + a.y) * P.dt);
        float2 x1 = make_float2(x.x + v1.x * P.dt, x.y + v1.y * P.dt);
        const float w1 = w + al * P.dt;
        bool c1 = false, c2 = false, c3 = false, c4 = false;
        if (x1.x > P.Lx - r) { x1.x = P.Lx - r; v1.x *= -eb; c1 = true; }
        if (x1.x < r) { x1.x = r; v1.x *= -eb; c2 = true; }
        if (x1.y > P.Ly - r) { x1.y = P.Ly - r; v1.y *= -eb; c3 = true; }
        if (x1.y < r) c4 = true;
        float2 lX = lamXin[id], lV = lamVin[id];
        float lW = lamWin[id];
        // floor contact (collideBoundary) and the final clamp of y
        if (c4) {
            lV.y *= -eb;  // vel.y *= -boundaryDamping
            lX.y = 0.0f;  // pos.y = radius
            using D = Dual<float, 7>;  // y, vx, vy, w, cn, mu, ktw
            const D py = seed<float, 7>(x1.y, 0), dvx = seed<float, 7>(v1.x, 1),
                    dvy = seed<float, 7>(v1.y, 2), dw = seed<float, 7>(w1, 3),
                    dcn = seed<float, 7>(P.cn[0], 4), dmu = seed<float, 7>(P.mu[0], 5),
                    dkt = seed<float, 7>(P.ktw[0], 6);
            D fx, fy, dm;
            unsigned fl;
            floor_law<D>(py, dvx, dvy, dw, D(r), D(-m * P.gravx), D(-m * P.gravy), dcn, dmu, dkt,
                         D(P.dt), fx, fy, dm, fl);
            // aw = F/m enters v (dt) and x (dt^2); alpha_w = r dm / I enters w (dt)
            const float lawx = lV.x * P.dt + lX.x * P.dt * P.dt;
            const float lawy = lV.y * P.dt + lX.y * P.dt * P.dt;
            const float lFx = lawx / m, lFy = lawy / m;
            const float lD = lW * P.dt * r / I;
            float g[7];
#pragma unroll
            for (int k = 0; k < 7; ++k) g[k] = fx.d[k] * lFx + fy.d[k] * lFy + dm.d[k] * lD;
            lX.y += g[0];
            lV.x += g[1];
            lV.y += g[2];
            lW += g[3];
            coef[4] += (double)g[4];
            coef[5] += (double)g[5];
            coef[6] += (double)g[6];
        }
        if (c3) { lX.y = 0.0f; lV.y *= -eb; }
        if (c2) { lX.x = 0.0f; lV.x *= -eb; }
        if (c1) { lX.x = 0.0f; lV.x *= -eb; }
        // x1 = x + v1 dt; v1 = v + (g + a) dt; w1 = w + alpha dt
        const float2 lV1 = make_float2(lV.x + lX.x * P.dt, lV.y + lX.y * P.dt);
        lx[i] = lX;
        lv[i] = lV1;
        lw[i] = lW;
        lamF[i] = make_float2(lV1.x * P.dt / m, lV1.y * P.dt / m);
        lamM[i] = lW * P.dt / I;
    }
    warp_add_coef(coef, seg, i, n, acc);
}

// Contacts of particle i in recorded step `rec`: adds the state cotangents
// of i to those of the integrate VJP (lx, lv, lw, sorted order) and writes
// the sums back to id order (lamX, lamV, lamW: nothing else reads or writes
// them while this kernel runs); once per pair (i < j), the coefficient
// cotangents.
__global__ void __launch_bounds__(kAdjThreads)
adj_pairs_kernel(KParams P0, const KParams* __restrict__ table, const uint32_t* __restrict__ spec,
                 StepRec rec0, RecSlot at, uint32_t n, const float2* __restrict__ lamF,
                 const float* __restrict__ lamM, const float2* __restrict__ lx,
                 const float2* __restrict__ lv, const float* __restrict__ lw,
                 float2* __restrict__ lamX, float2* __restrict__ lamV, float* __restrict__ lamW,
                 double* __restrict__ acc) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double coef[kCoef] = {0, 0, 0, 0, 0, 0, 0};
    const uint32_t seg = i < n ? (table ? spec[i] : 0u) : 0xffffffffu;
    if (i < n) {
        const StepRec rec = rec_at(rec0, at);
        const KParams& P = table ? table[seg] : P0;
        const float2 p = rec.pos[i], v = rec.vel[i];
        const float w = rec.omega[i], r = rec.radius[i];
        const float2 lFi = lamF[i];
        const float lMi = lamM[i];
        const float4 pc = P.pair[0];
        const int2 g = grid_pos(P, p);
        float gx = 0, gy = 0, gvx = 0, gvy = 0, gw = 0;
        for (int dy = -1; dy <= 1; ++dy) {
            for (int dx = -1; dx <= 1; ++dx) {
                const uint2 se = rec.cells[grid_hash(P, g.x + dx, g.y + dy)];
                const uint32_t end = se.x < se.y ? se.y : 0u;
                for (uint32_t j = se.x < se.y ? se.x : 0u; j < end; ++j) {
                    if (j == i) continue;
                    const float2 q = rec.pos[j];
                    const float rj = rec.radius[j];
                    const float rx = q.x - p.x, ry = q.y - p.y;
                    const float d2 = rx * rx + ry * ry;
                    const float cd = r + rj;
                    if (!(d2 <= cd * cd * 1.000002f && sqrtf(d2) < cd)) continue;
                    const float2 vj = rec.vel[j];
                    const float wj = rec.omega[j];
                    const float2 lFj = lamF[j];
                    const float wfx = lFi.x - lFj.x, wfy = lFi.y - lFj.y;
                    const float wd = lMi * r + lamM[j] * rj;
                    {   // derivatives with respect to particle i's state
                        using D = Dual<float, 5>;
                        D fx, fy, dm;
                        unsigned fl;
                        pair_law<D>(seed<float, 5>(p.x, 0), seed<float, 5>(p.y, 1), D(q.x), D(q.y),
                                    seed<float, 5>(v.x, 2), seed<float, 5>(v.y, 3), D(vj.x),
                                    D(vj.y), seed<float, 5>(w, 4), D(wj), D(r), D(rj), D(pc.x),
                                    D(pc.y), D(pc.z), D(pc.w), D(P.dt), fx, fy, dm, fl);
                        gx += fx.d[0] * wfx + fy.d[0] * wfy + dm.d[0] * wd;
                        gy += fx.d[1] * wfx + fy.d[1] * wfy + dm.d[1] * wd;
                        gvx += fx.d[2] * wfx + fy.d[2] * wfy + dm.d[2] * wd;
                        gvy += fx.d[3] * wfx + fy.d[3] * wfy + dm.d[3] * wd;
                        gw += fx.d[4] * wfx + fy.d[4] * wfy + dm.d[4] * wd;
                    }
                    if (i < j) {  // coefficients: once per pair
                        using D = Dual<float, 4>;
                        D fx, fy, dm;
                        unsigned fl;
                        pair_law<D>(D(p.x), D(p.y), D(q.x), D(q.y), D(v.x), D(v.y), D(vj.x),
                                    D(vj.y), D(w), D(wj), D(r), D(rj), seed<float, 4>(pc.x, 0),
                                    seed<float, 4>(pc.y, 1), seed<float, 4>(pc.z, 2),
                                    seed<float, 4>(pc.w, 3), D(P.dt), fx, fy, dm, fl);
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            coef[k] += (double)fx.d[k] * wfx + (double)fy.d[k] * wfy +
                                       (double)dm.d[k] * wd;
                    }
                }
            }
        }
        const uint32_t k = rec.id[i];
        const float2 l = lx[i], u = lv[i];
        lamX[k] = make_float2(l.x + gx, l.y + gy);
        lamV[k] = make_float2(u.x + gvx, u.y + gvy);
        lamW[k] = lw[i] + gw;
    }
    warp_add_coef(coef, seg, i, n, acc);
}

// Per specimen s: the sum of acc[k * n + slot] over its slots
// [first[s], first[s + 1]), in a fixed order (strided per thread, then a
// fixed-shape block reduction).
constexpr int kSumThreads = 256;
__global__ void __launch_bounds__(kSumThreads)
adj_coef_sum_kernel(const double* __restrict__ acc, uint32_t n, const uint32_t* __restrict__ first,
                    double* __restrict__ out) {
    __shared__ double red[kSumThreads / 32];
    const uint32_t s = blockIdx.x;
    const uint32_t a = first ? first[s] : 0u, b = first ? first[s + 1] : n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < kCoef; ++k) {
        double x = 0.0;
        for (uint32_t j = a + threadIdx.x; j < b; j += kSumThreads) x += acc[(size_t)k * n + j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) red[warp] = x;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < kSumThreads / 32; ++w) t += red[w];
            out[(size_t)s * kCoef + k] = t;
        }
        __syncthreads();
    }
}

}  // namespace

size_t adj_step_bytes(uint32_t n, uint32_t numCells) {
    return 4 * al256(8ull * n) + 4 * al256(4ull * n) + al256(4ull * n) + al256(8ull * numCells);
}

StepRec carve_step(void* base, uint32_t n, uint32_t numCells) {
    char* p = static_cast<char*>(base);
    StepRec r;
    r.pos = reinterpret_cast<float2*>(p); p += al256(8ull * n);
    r.vel = reinterpret_cast<float2*>(p); p += al256(8ull * n);
    r.acc = reinterpret_cast<float2*>(p); p += al256(8ull * n);
    p += al256(8ull * n);  // spare, keeps the layout of adj_step_bytes
    r.omega = reinterpret_cast<float*>(p); p += al256(4ull * n);
    r.radius = reinterpret_cast<float*>(p); p += al256(4ull * n);
    r.mass = reinterpret_cast<float*>(p); p += al256(4ull * n);
    r.alpha = reinterpret_cast<float*>(p); p += al256(4ull * n);
    r.id = reinterpret_cast<uint32_t*>(p); p += al256(4ull * n);
    r.cells = reinterpret_cast<uint2*>(p);
    return r;
}

namespace {
__global__ void __launch_bounds__(kAdjThreads)
adj_record_kernel(StepRec r0, RecSlot at, DynSet d, StatSet s, const uint32_t* __restrict__ src,
                  const uint2* __restrict__ cells,
                  const float2* __restrict__ acc, const float* __restrict__ alpha, uint32_t n,
                  uint32_t numCells) {
    const StepRec r = rec_at(r0, at);
    const uint32_t m = n > numCells ? n : numCells;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        if (i < n) {
            const uint32_t si = src[i];
            r.pos[i] = d.pos[i];
            r.vel[i] = d.vel[si];
            r.omega[i] = d.omega[si];
            r.radius[i] = s.radius[i];
            r.mass[i] = s.mass[si];
            r.id[i] = s.id[si];
            r.acc[i] = acc[i];
            r.alpha[i] = alpha[i];
        }
        if (i < numCells) r.cells[i] = cells[i];
    }
}
}  // namespace

cudaError_t adj_record_step(void* recBase, RecSlot at, uint32_t n, uint32_t numCells, DynSet d,
                            StatSet s, const uint32_t* src, const uint2* cells, const float2* acc,
                            const float* alpha, cudaStream_t st) {
    const uint32_t m = n > numCells ? n : numCells;
    const unsigned b = std::min<unsigned>(blocks_for(m, kAdjThreads), 148u * 16u);
    adj_record_kernel<<<b, kAdjThreads, 0, st>>>(carve_step(recBase, n, numCells), at, d, s, src,
                                                 cells, acc, alpha, n, numCells);
    return cudaGetLastError();
}

cudaError_t adj_backward_step(const KParams& P, const KParams* table, const uint32_t* spec,
                              void* recBase, RecSlot at, uint32_t n, uint32_t numCells,
                              float2* lamX, float2* lamV, float* lamW, float2* tlx, float2* tlv,
                              float* tlw, float2* lamF, float* lamM, double* acc, cudaStream_t st) {
    const StepRec rec = carve_step(recBase, n, numCells);
    const unsigned b = blocks_for(n, kAdjThreads);
    adj_integrate_kernel<<<b, kAdjThreads, 0, st>>>(P, table, spec, rec, at, n, lamX, lamV, lamW,
                                                    tlx, tlv, tlw, lamF, lamM, acc);
    adj_pairs_kernel<<<b, kAdjThreads, 0, st>>>(P, table, spec, rec, at, n, lamF, lamM, tlx, tlv,
                                                tlw, lamX, lamV, lamW, acc);
    return cudaGetLastError();
}

cudaError_t adj_sum_coef(const double* acc, uint32_t n, const uint32_t* first, uint32_t numSpecimens,
                         double* out, cudaStream_t st) {
    adj_coef_sum_kernel<<<numSpecimens, kSumThreads, 0, st>>>(acc, n, first, out);
    return cudaGetLastError();
}

size_t adj_acc_bytes(uint32_t n) { return sizeof(double) * kCoef * (size_t)n; }

}  // namespace dem
