// Shared device code for the DEM step: launch parameters, the uniform-grid
// hash and the contact law.
//
// Every expression here spells the reference's floating-point operations in
// the reference's order (src/particles_kernel.cuh).  The library is compiled
// with -fmad=false and IEEE division/square root, so each float operation is
// one correctly rounded IEEE operation, exactly as in a host build of the
// reference without FP contraction; results are therefore bit-identical to
// that build, stage by stage.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/demso_b200.h"

namespace dem {

constexpr uint32_t kEmptyCell = 0xffffffffu;
// Largest arrival group / leaving cell the incremental sort scans per particle;
// anything larger sends the next step to the full radix sort.
constexpr uint32_t kMaxGroup = 64;
constexpr int kMaxMat = DEM_MAX_MATERIALS;

// Launch-time parameters, passed by value (lives in the kernel-parameter
// constant bank, so contexts are independent and graph capture is trivial).
struct KParams {
    uint32_t n;
    uint32_t gx, gy;      // powers of two
    uint32_t nmat;
    float gxf, gyf;       // (float)gx, (float)gy as the reference's uint->float conversion
    float Lx, Ly;
    float dt;
    float gravx, gravy;
    float ktWall;
    // per material
    float cn[kMaxMat];    // normalDamping (wall dashpot uses the material's own value)
    float eb[kMaxMat];    // boundaryDamping
    float mu[kMaxMat];    // frictionCoefficient
    float ktw[kMaxMat];   // seriesAssociation(shearStiffness, boundaryShearStiffness)
    float at[kMaxMat];    // attractCoefficient
    // per material pair (a * nmat + b): series kn, series kt, series cn, mean mu
    float4 pair[kMaxMat * kMaxMat];
    // Neighbour culling (context step only): an upper bound on every radius
    // (INFINITY disables culling), the cell size, and an absolute margin that
    // covers float rounding of positions and cell bounds.
    float rmax;
    float cellW, cellH;
    float cullMargin;
    float invLx, invLy;  // rn(1/Lx), rn(1/Ly) for grid_pos_fast
    // Batched form: the specimen's first cell in the global cell numbering (0
    // for a single scene), log2(gx), and whether culling is valid here.
    uint32_t cellOff;
    uint32_t log2gx;
    uint32_t cull;
    // Row window: the context's cell rows are the scene's rows rowOff,
    // rowOff + 1, ... (gy of them, wrapping); gyf, Ly, cellH and invLy stay
    // the whole scene's, so positions give the scene's rows bit for bit.
    // 0 for a context over the whole grid and for every batch.
    int32_t rowOff;
};

// particles_kernel.cuh:36-41, evaluated on the host when KParams is built.
static inline __host__ __device__ float series_assoc(float a, float b) {
    if (a == 0.0f || b == 0.0f) return 0.0f;
    return (a * b) / (a + b);
}

__device__ __forceinline__ float len2(float x, float y) { return sqrtf(x * x + y * y); }

// main.cu:193 -- inertia of a disk as the reference writes it: 2 m r^2 / 5.
__device__ __forceinline__ float inertia_of(float m, float r) { return 2.0f * m * r * r / 5.0f; }

// particles_kernel.cuh:114-121: float multiply by the grid size, IEEE divide by
// the box size, floor, truncate to int.
__device__ __forceinline__ int2 grid_pos(const KParams& P, float2 p) {
    int2 g;
    g.x = (int)floorf(p.x * P.gxf / P.Lx);
    g.y = (int)floorf(p.y * P.gyf / P.Ly);
    return g;
}

// grid_pos without the two divisions in the common case.  The reference's
// quotient q = rn(rn(p * g) / L) and t * rn(1/L) (t = rn(p * g)) differ by at
// most 3 ulp of q (two roundings of the product, one of the reciprocal, one
// of the quotient: 4 * 2^-24 relative), so floor() of both agrees unless
// t * rn(1/L) lies within 2^-20 * |q| of an integer; then, and for
// non-finite or huge values, the IEEE division decides.
__device__ __forceinline__ int grid_axis_fast(float p, float gf, float L, float invL) {
    const float t = p * gf;
    const float qa = t * invL;
    const float fl = floorf(qa);
    const float tol = fabsf(qa) * 9.5367431640625e-07f;  // 2^-20
    if (fabsf(qa) < 8388608.0f && qa - fl > tol && (fl + 1.0f) - qa > tol) return (int)fl;
    return (int)floorf(t / L);
}
__device__ __forceinline__ int2 grid_pos_fast(const KParams& P, float2 p) {
    return make_int2(grid_axis_fast(p.x, P.gxf, P.Lx, P.invLx),
                     grid_axis_fast(p.y, P.gyf, P.Ly, P.invLy));
}

// particles_kernel.cuh:124-130: power-of-two wrap, row-major cell index, for
// a cell given in the context's own rows (a key's decoded row and its
// neighbours).
__device__ __forceinline__ uint32_t cell_index(const KParams& P, int x, int y) {
    x &= (int)(P.gx - 1u);
    y &= (int)(P.gy - 1u);
    return P.cellOff + (uint32_t)y * P.gx + (uint32_t)x;
}

// The same for a cell given in the scene's rows (grid_pos of a position): a
// row window first moves the row to its own numbering.
__device__ __forceinline__ uint32_t grid_hash(const KParams& P, int x, int y) {
    return cell_index(P, x, y - P.rowOff);
}

// `pressure += length(force) / (4*M_PI*r*r)` -- the reference does this sum in
// double and stores the float result.
__device__ __forceinline__ float add_pressure(float pr, float flen, float r) {
    const double den = 4.0 * 3.14159265358979323846 * (double)r * (double)r;
    return (float)((double)pr + (double)flen / den);
}

// One particle pair, particles_kernel.cuh:236-307 (collideSpheres).  A is the
// particle being updated, B the neighbour.  Returns the force on A; adds the
// moment and the pressure contribution.
__device__ __forceinline__ float2 pair_force(float2 pA, float2 pB, float2 vA, float2 vB, float wA,
                                             float wB, float rA, float rB, float4 pc, float dt,
                                             float& moment, float& pressure) {
    const float relx = pB.x - pA.x, rely = pB.y - pA.y;
    const float dist = len2(relx, rely);
    const float cd = rA + rB;
    float2 f = make_float2(0.0f, 0.0f);
    if (dist < cd) {
        const float nx = relx / dist, ny = rely / dist;
        const float tx = -ny, ty = nx;
        const float rvx = vB.x - vA.x, rvy = vB.y - vA.y;
        const float vn = rvx * nx + rvy * ny;
        const float vtx = rvx - vn * nx, vty = rvy - vn * ny;
        const float fs = -pc.x * (cd - dist);
        f.x = fs * nx;
        f.y = fs * ny;
        if (vn < 0.0f) {
            const float c = pc.z * vn;
            f.x += c * nx;
            f.y += c * ny;
        }
        pressure = add_pressure(pressure, len2(f.x, f.y), rA);
        if (pc.w != 0.0f) {
            const float sw = rA * wA + rB * wB;
            const float vcx = vtx - sw * tx, vcy = vty - sw * ty;
            const float ftrx = pc.y * vcx * dt, ftry = pc.y * vcy * dt;
            const float ftmax = pc.w * len2(f.x, f.y);
            float ftx, fty;
            if (len2(ftrx, ftry) < ftmax) {
                ftx = ftrx;
                fty = ftry;
            } else {
                const float l = len2(vcx, vcy);
                ftx = ftmax * vcx / l;
                fty = ftmax * vcy / l;
            }
            f.x += ftx;
            f.y += fty;
            moment += rA * (ftx * tx + fty * ty);
        }
    }
    return f;
}

// particles_kernel.cuh:311-342 (attractSpheres), only compiled into the
// attraction variants of the collide kernels.
__device__ __forceinline__ float2 pair_attract(float2 pA, float2 pB, float rA, float rB, float aA,
                                               float aB, float& pressure) {
    const float relx = pB.x - pA.x, rely = pB.y - pA.y;
    const float dist = len2(relx, rely);
    const float dA = (float)((double)(rA * 2.0f) * 1.2);
    const float dB = (float)((double)(rB * 2.0f) * 1.2);
    const float nx = relx / dist, ny = rely / dist;
    float2 f = make_float2(0.0f, 0.0f);
    if (dist < dA) {
        const float c = aA * (dA - dist);
        f.x += c * nx;
        f.y += c * ny;
    }
    if (dist < dB) {
        const float c = aB * (dB - dist);
        f.x += c * nx;
        f.y += c * ny;
    }
    pressure = add_pressure(pressure, len2(f.x, f.y), rA);
    return f;
}

// Floor contact, particles_kernel.cuh:388-456 (collideBoundary with the
// boundary point (x, 0)).  Returns the wall acceleration; adds to alpha and
// pressure.
__device__ __forceinline__ float2 floor_contact(const KParams& P, float2 p, float2 v, float w,
                                                float r, float m, uint32_t mat, float& walpha,
                                                float& pressure) {
    const float relx = p.x - p.x, rely = 0.0f - p.y;
    const float dist = len2(relx, rely);
    float fx = 0.0f, fy = 0.0f;
    if (dist < r) {
        const float nx = relx / dist, ny = rely / dist;
        const float tx = -ny, ty = nx;
        const float rvx = -v.x, rvy = -v.y;
        const float vn = rvx * nx + rvy * ny;
        const float vtx = rvx - vn * nx, vty = rvy - vn * ny;
        const float kt = P.ktw[mat];
        const float nm = -m;
        fx = nm * P.gravx;
        fy = nm * P.gravy;
        if (vn < 0.0f) {
            const float c = P.cn[mat] * vn;
            fx += c * nx;
            fy += c * ny;
        }
        pressure = add_pressure(pressure, len2(fx, fy), r);
        const float mu = P.mu[mat];
        if (mu != 0.0f) {
            const float rw = r * w;
            const float vcx = vtx - rw * tx, vcy = vty - rw * ty;
            const float ftrx = kt * vcx * P.dt, ftry = kt * vcy * P.dt;
            const float ftmax = mu * len2(fx, fy);
            float ftx, fty;
            if (len2(ftrx, ftry) < ftmax) {
                ftx = ftrx;
                fty = ftry;
            } else {
                const float l = len2(vcx, vcy);
                ftx = ftmax * vcx / l;
                fty = ftmax * vcy / l;
            }
            fx = ftx;
            fy = fty;
            walpha += r * (ftx * tx + fty * ty) / inertia_of(m, r);
        }
    }
    return make_float2(fx / m, fy / m);
}

// Integration of one particle, particles_kernel.cuh:580-627
// (integrateSystemD): symplectic Euler, theta wrap in double, side/top walls
// as position clamps, floor through floor_contact.
struct Dyn {
    float2 p, v;
    float th, w;
};

__device__ __forceinline__ void integrate_one(const KParams& P, Dyn& s, float2 a, float al, float r,
                                              float m, uint32_t mat, float& pressure) {
    s.v.x += (P.gravx + a.x) * P.dt;
    s.v.y += (P.gravy + a.y) * P.dt;
    s.p.x += s.v.x * P.dt;
    s.p.y += s.v.y * P.dt;
    s.w += al * P.dt;
    s.th += s.w * P.dt;
    const double twopi = 2.0 * 3.14159265358979323846;
    // (double)th > 2*pi exactly when th > 6.2831850f, the largest float below
    // 2*pi (the next float up, 6.28318548f, is above it)
    if (s.th > 6.28318500518798828125f)
        s.th = (float)((double)s.th - twopi * floor((double)s.th / twopi));
    if (s.th < 0.0f) s.th = (float)((double)s.th - twopi * floor((double)s.th / twopi));
    const float eb = P.eb[mat];
    if (s.p.x > P.Lx - r) { s.p.x = P.Lx - r; s.v.x *= -eb; }
    if (s.p.x < r) { s.p.x = r; s.v.x *= -eb; }
    if (s.p.y > P.Ly - r) { s.p.y = P.Ly - r; s.v.y *= -eb; }
    if (s.p.y < r) {
        float wa = 0.0f;
        const float2 aw = floor_contact(P, s.p, s.v, s.w, r, m, mat, wa, pressure);
        s.v.x += aw.x * P.dt;
        s.v.y += aw.y * P.dt;
        s.p.x += aw.x * P.dt * P.dt;
        s.p.y += aw.y * P.dt * P.dt;
        s.w += wa * P.dt;
        s.th += wa * P.dt * P.dt;
        s.p.y = r;
        s.v.y *= -eb;
    }
}

}  // namespace dem
