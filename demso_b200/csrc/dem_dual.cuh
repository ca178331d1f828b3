// Forward-mode dual numbers and the contact law written once for any scalar
// type, for the adjoint.  Dual<T, N> carries a value and N partial
// derivatives; evaluating the contact law on duals seeded with unit tangents
// gives its Jacobian, whose transpose the adjoint applies.
//
// The law below is the reference's (particles_kernel.cuh:236-307 for a pair,
// :388-456 for the floor) without the pressure diagnostic, with every branch
// decided by the primal values exactly as the forward decides it.
#pragma once

#include <cuda_runtime.h>

namespace dem {

template <typename T, int N>
struct Dual {
    T v;
    T d[N];
    __host__ __device__ Dual() : v(0) {
#pragma unroll
        for (int k = 0; k < N; ++k) d[k] = T(0);
    }
    __host__ __device__ Dual(T x) : v(x) {
#pragma unroll
        for (int k = 0; k < N; ++k) d[k] = T(0);
    }
};

template <typename T, int N>
__host__ __device__ inline Dual<T, N> seed(T x, int k) {
    Dual<T, N> r(x);
    r.d[k] = T(1);
    return r;
}

#define DEM_DUAL_BIN(OP, VEXPR, DEXPR)                                                      \
    template <typename T, int N>                                                            \
    __host__ __device__ inline Dual<T, N> operator OP(const Dual<T, N>& a,                  \
                                                      const Dual<T, N>& b) {                \
        Dual<T, N> r;                                                                       \
        r.v = VEXPR;                                                                        \
        _Pragma("unroll") for (int k = 0; k < N; ++k) r.d[k] = DEXPR;                      \
        return r;                                                                           \
    }
DEM_DUAL_BIN(+, a.v + b.v, a.d[k] + b.d[k])
DEM_DUAL_BIN(-, a.v - b.v, a.d[k] - b.d[k])
DEM_DUAL_BIN(*, a.v * b.v, a.d[k] * b.v + a.v * b.d[k])
#undef DEM_DUAL_BIN

template <typename T, int N>
__host__ __device__ inline Dual<T, N> operator/(const Dual<T, N>& a, const Dual<T, N>& b) {
    Dual<T, N> r;
    r.v = a.v / b.v;
    const T ib = T(1) / b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}

template <typename T, int N>
__host__ __device__ inline Dual<T, N> operator-(const Dual<T, N>& a) {
    Dual<T, N> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
    return r;
}

template <typename T, int N>
__host__ __device__ inline Dual<T, N> dsqrt(const Dual<T, N>& a) {
    Dual<T, N> r;
    r.v = sqrt(a.v);
    const T h = r.v > T(0) ? T(0.5) / r.v : T(0);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * h;
    return r;
}

template <typename T>
__host__ __device__ inline T value_of(T x) { return x; }
template <typename T, int N>
__host__ __device__ inline T value_of(const Dual<T, N>& x) { return x.v; }

__host__ __device__ inline float dsqrt(float a) { return sqrtf(a); }
__host__ __device__ inline double dsqrt(double a) { return sqrt(a); }

// Pair law for A (the particle updated) against B.  Outputs the force on A
// and the moment arm product d = Ft . t (A's moment is rA * d).  flags: bit0
// contact, bit1 dashpot active (vn < 0), bit2 friction evaluated (mu != 0),
// bit3 slip (|Ftr| >= Ftmax).
template <typename S>
__host__ __device__ inline void pair_law(S pAx, S pAy, S pBx, S pBy, S vAx, S vAy, S vBx, S vBy,
                                         S wA, S wB, S rA, S rB, S kn, S kt, S cn, S mu, S dt,
                                         S& fx, S& fy, S& dmom, unsigned& flags) {
    const S relx = pBx - pAx, rely = pBy - pAy;
    const S dist = dsqrt(relx * relx + rely * rely);
    const S cd = rA + rB;
    fx = S(0);
    fy = S(0);
    dmom = S(0);
    flags = 0;
    if (!(value_of(dist) < value_of(cd))) return;
    flags |= 1u;
    const S nx = relx / dist, ny = rely / dist;
    const S tx = -ny, ty = nx;
    const S rvx = vBx - vAx, rvy = vBy - vAy;
    const S vn = rvx * nx + rvy * ny;
    const S vtx = rvx - vn * nx, vty = rvy - vn * ny;
    const S fs = -kn * (cd - dist);
    fx = fs * nx;
    fy = fs * ny;
    if (value_of(vn) < 0) {
        flags |= 2u;
        const S c = cn * vn;
        fx = fx + c * nx;
        fy = fy + c * ny;
    }
    if (value_of(mu) != 0) {
        flags |= 4u;
        const S sw = rA * wA + rB * wB;
        const S vcx = vtx - sw * tx, vcy = vty - sw * ty;
        const S ftrx = kt * vcx * dt, ftry = kt * vcy * dt;
        const S ftmax = mu * dsqrt(fx * fx + fy * fy);
        S ftx, fty;
        if (value_of(dsqrt(ftrx * ftrx + ftry * ftry)) < value_of(ftmax)) {
            ftx = ftrx;
            fty = ftry;
        } else {
            flags |= 8u;
            const S l = dsqrt(vcx * vcx + vcy * vcy);
            ftx = ftmax * vcx / l;
            fty = ftmax * vcy / l;
        }
        fx = fx + ftx;
        fy = fy + fty;
        dmom = ftx * tx + fty * ty;
    }
}

// Floor law (collideBoundary against (x, 0)): the wall force and moment of
// a particle below y = r.  gm = (-m * gx, -m * gy).  Returns the force and
// Ft . t; the caller divides by m and I.  flags: bit0 contact, bit1 dashpot,
// bit2 friction, bit3 slip.
template <typename S>
__host__ __device__ inline void floor_law(S py, S vx, S vy, S w, S r, S gmx, S gmy, S cn, S mu,
                                          S ktw, S dt, S& fx, S& fy, S& dmom, unsigned& flags) {
    const S relx = S(0), rely = S(0) - py;
    const S dist = dsqrt(relx * relx + rely * rely);
    fx = S(0);
    fy = S(0);
    dmom = S(0);
    flags = 0;
    if (!(value_of(dist) < value_of(r))) return;
    flags |= 1u;
    const S nx = relx / dist, ny = rely / dist;
    const S tx = -ny, ty = nx;
    const S rvx = -vx, rvy = -vy;
    const S vn = rvx * nx + rvy * ny;
    const S vtx = rvx - vn * nx, vty = rvy - vn * ny;
    fx = gmx;
    fy = gmy;
    if (value_of(vn) < 0) {
        flags |= 2u;
        const S c = cn * vn;
        fx = fx + c * nx;
        fy = fy + c * ny;
    }
    if (value_of(mu) != 0) {
        flags |= 4u;
        const S rw = r * w;
        const S vcx = vtx - rw * tx, vcy = vty - rw * ty;
        const S ftrx = ktw * vcx * dt, ftry = ktw * vcy * dt;
        const S ftmax = mu * dsqrt(fx * fx + fy * fy);
        S ftx, fty;
        if (value_of(dsqrt(ftrx * ftrx + ftry * ftry)) < value_of(ftmax)) {
            ftx = ftrx;
            fty = ftry;
        } else {
            flags |= 8u;
            const S l = dsqrt(vcx * vcx + vcy * vcy);
            ftx = ftmax * vcx / l;
            fty = ftmax * vcy / l;
        }
        fx = ftx;
        fy = fty;
        dmom = ftx * tx + fty * ty;
    }
}

}  // namespace dem
