/* Test infrastructure (oracle only) -- never linked into the product.
 *
 * Forward-mode tangent of the oracle step: the same step as dem_oracle.c
 * (calc_hash, stable sort, reorder, collide, integrate in the order of
 * main.cu:431-507), evaluated on numbers that carry a value and K = 4
 * directional derivatives.  The values follow exactly the operations of
 * dem_oracle.c, so the primal trajectory and the branch signature equal the
 * oracle's at the same precision; the derivatives are the exact derivatives
 * of that piecewise-smooth trajectory along each seeded direction (the
 * "frozen branch" derivative an adjoint computes).
 *
 * Built twice like the oracle: B = double (libdem_tangent_f64.so, the FP64
 * oracle adjoint against which the GPU adjoint is checked) and B = float
 * (libdem_tangent_f32.so, the same derivative along the float trajectory the
 * GPU forward follows).  The attraction law is not differentiated; the entry
 * point refuses materials with a nonzero attraction coefficient.
 *
 * Differentiated inputs: the material coefficients (normal / shear
 * stiffness, normal damping, friction), the wall stiffnesses and the initial
 * positions, velocities and spins.  Radius, mass, boundary damping, gravity
 * and dt are constants.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "dem_oracle.h"

namespace {

constexpr int K = 4;

template <typename B>
struct T {
    B v;
    B d[K];
    T() : v(0) { for (int k = 0; k < K; ++k) d[k] = 0; }
    T(B x) : v(x) { for (int k = 0; k < K; ++k) d[k] = 0; }
};

template <typename B> T<B> operator+(const T<B>& a, const T<B>& b) {
    T<B> r; r.v = a.v + b.v;
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <typename B> T<B> operator-(const T<B>& a, const T<B>& b) {
    T<B> r; r.v = a.v - b.v;
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <typename B> T<B> operator-(const T<B>& a) {
    T<B> r; r.v = -a.v;
    for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
    return r;
}
template <typename B> T<B> operator*(const T<B>& a, const T<B>& b) {
    T<B> r; r.v = a.v * b.v;
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <typename B> T<B> operator/(const T<B>& a, const T<B>& b) {
    T<B> r; r.v = a.v / b.v;
    for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] * b.v - a.v * b.d[k]) / (b.v * b.v);
    return r;
}
template <typename B> T<B> tsqrt(const T<B>& a) {
    T<B> r; r.v = std::sqrt(a.v);
    for (int k = 0; k < K; ++k) r.d[k] = r.v > 0 ? a.d[k] / (B(2) * r.v) : B(0);
    return r;
}

template <typename B> struct V2 { T<B> x, y; };
template <typename B> V2<B> v2(const T<B>& x, const T<B>& y) { V2<B> r; r.x = x; r.y = y; return r; }
template <typename B> T<B> dot(const V2<B>& a, const V2<B>& b) { return a.x * b.x + a.y * b.y; }
template <typename B> T<B> len(const V2<B>& a) { return tsqrt(dot(a, a)); }

/* Branch signature, mixed exactly as dem_oracle.c mixes it. */
uint64_t g_sig;
inline void sig_mix(uint64_t v) { g_sig = (g_sig ^ v) * 1099511628211ull; }

template <typename B>
struct Mat { T<B> kn, kt, cn, mu; B eb; };

template <typename B>
struct Sys {
    B Lx, Ly, dt, gx_f, gy_f, gravx, gravy;
    uint32_t gx, gy;
    T<B> ktWall;
    Mat<B> m;
};

/* particles_kernel.cuh:36-41 */
template <typename B> T<B> series(const T<B>& a, const T<B>& b) {
    if (a.v == 0 || b.v == 0) return T<B>(0);
    return (a * b) / (a + b);
}

/* main.cu:193 */
template <typename B> T<B> inertia(B m, B r) { return T<B>(B(2) * m * r * r / B(5)); }

template <typename B> void grid_pos(const Sys<B>& s, B px, B py, int* gx, int* gy) {
    *gx = (int)std::floor(px * s.gx_f / s.Lx);
    *gy = (int)std::floor(py * s.gy_f / s.Ly);
}
template <typename B> uint32_t grid_hash(const Sys<B>& s, int x, int y) {
    x &= (int)(s.gx - 1);
    y &= (int)(s.gy - 1);
    return (uint32_t)y * s.gx + (uint32_t)x;
}

template <typename B>
struct State {
    std::vector<V2<B>> pos, vel;
    std::vector<T<B>> omega;
    std::vector<B> theta, radius, mass;
    std::vector<uint32_t> id;
};

/* particles_kernel.cuh:236-307 (collideSpheres), one material */
template <typename B>
V2<B> collide_spheres(const Sys<B>& s, const V2<B>& pA, const V2<B>& pB, const V2<B>& vA,
                      const V2<B>& vB, const T<B>& wA, const T<B>& wB, B rA, B rB,
                      T<B>& moment) {
    const V2<B> rel = v2(pB.x - pA.x, pB.y - pA.y);
    const T<B> dist = len(rel);
    const T<B> cd = T<B>(rA + rB);
    V2<B> force = v2(T<B>(0), T<B>(0));
    if (dist.v < cd.v) {
        const V2<B> nrm = v2(rel.x / dist, rel.y / dist);
        const V2<B> tng = v2(-nrm.y, nrm.x);
        const V2<B> rv = v2(vB.x - vA.x, vB.y - vA.y);
        const T<B> vn = dot(rv, nrm);
        const V2<B> vt = v2(rv.x - vn * nrm.x, rv.y - vn * nrm.y);
        const T<B> kn = series(s.m.kn, s.m.kn);
        const T<B> kt = series(s.m.kt, s.m.kt);
        const T<B> cn = series(s.m.cn, s.m.cn);
        const T<B> mu = (s.m.mu + s.m.mu) / T<B>(2);
        const T<B> fs = -kn * (cd - dist);
        force = v2(fs * nrm.x, fs * nrm.y);
        if (vn.v < 0) {
            const T<B> c = cn * vn;
            force.x = force.x + c * nrm.x;
            force.y = force.y + c * nrm.y;
        }
        uint64_t br = 1u | (vn.v < 0 ? 2u : 0u);
        if (mu.v != 0) {
            const T<B> sw = T<B>(rA) * wA + T<B>(rB) * wB;
            const V2<B> vc = v2(vt.x - sw * tng.x, vt.y - sw * tng.y);
            const V2<B> ftr = v2(kt * vc.x * T<B>(s.dt), kt * vc.y * T<B>(s.dt));
            const T<B> ftmax = mu * len(force);
            V2<B> ft;
            if (len(ftr).v < ftmax.v) {
                ft = ftr;
            } else {
                const T<B> l = len(vc);
                ft = v2(ftmax * vc.x / l, ftmax * vc.y / l);
                br |= 4u;
            }
            force.x = force.x + ft.x;
            force.y = force.y + ft.y;
            moment = moment + T<B>(rA) * dot(ft, tng);
        }
        sig_mix(br);
    }
    return force;
}

/* particles_kernel.cuh:388-456 (collideBoundary) against the floor point (x, 0) */
template <typename B>
V2<B> collide_floor(const Sys<B>& s, const V2<B>& p, const V2<B>& v, const T<B>& w, B r, B m,
                    T<B>& walpha) {
    const V2<B> rel = v2(p.x - p.x, T<B>(0) - p.y);
    const T<B> dist = len(rel);
    V2<B> force = v2(T<B>(0), T<B>(0));
    if (dist.v < r) {
        const V2<B> nrm = v2(rel.x / dist, rel.y / dist);
        const V2<B> tng = v2(-nrm.y, nrm.x);
        const V2<B> rv = v2(-v.x, -v.y);
        const T<B> vn = dot(rv, nrm);
        const V2<B> vt = v2(rv.x - vn * nrm.x, rv.y - vn * nrm.y);
        const T<B> kt = series(s.m.kt, s.ktWall);
        const T<B> cn = s.m.cn;
        const B nm = -m;
        force = v2(T<B>(nm * s.gravx), T<B>(nm * s.gravy));
        if (vn.v < 0) {
            const T<B> c = cn * vn;
            force.x = force.x + c * nrm.x;
            force.y = force.y + c * nrm.y;
        }
        if (s.m.mu.v != 0) {
            const T<B> rw = T<B>(r) * w;
            const V2<B> vc = v2(vt.x - rw * tng.x, vt.y - rw * tng.y);
            const V2<B> ftr = v2(kt * vc.x * T<B>(s.dt), kt * vc.y * T<B>(s.dt));
            const T<B> ftmax = s.m.mu * len(force);
            V2<B> ft;
            if (len(ftr).v < ftmax.v) {
                ft = ftr;
            } else {
                const T<B> l = len(vc);
                ft = v2(ftmax * vc.x / l, ftmax * vc.y / l);
            }
            force = ft;
            walpha = walpha + T<B>(r) * dot(ft, tng) / inertia(m, r);
        }
    }
    return v2(force.x / T<B>(m), force.y / T<B>(m));
}

template <typename B>
void step(const Sys<B>& s, State<B>& a, State<B>& b, uint64_t* sig) {
    const uint32_t n = (uint32_t)a.pos.size();
    const uint32_t cells = s.gx * s.gy;
    /* calc_hash + stable sort + reorder (particles_kernel.cuh:133-233,
     * functions.cu:336-371) */
    std::vector<uint32_t> hash(n), order(n);
    for (uint32_t i = 0; i < n; ++i) {
        int x, y;
        grid_pos(s, a.pos[i].x.v, a.pos[i].y.v, &x, &y);
        hash[i] = grid_hash(s, x, y);
    }
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t p, uint32_t q) { return hash[p] < hash[q]; });
    std::vector<uint32_t> cellStart(cells, 0xffffffffu), cellEnd(cells, 0u);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t src = order[i], h = hash[src];
        if (i == 0 || h != hash[order[i - 1]]) {
            cellStart[h] = i;
            if (i > 0) cellEnd[hash[order[i - 1]]] = i;
        }
        if (i == n - 1) cellEnd[h] = i + 1;
        b.pos[i] = a.pos[src];
        b.vel[i] = a.vel[src];
        b.theta[i] = a.theta[src];
        b.omega[i] = a.omega[src];
        b.radius[i] = a.radius[src];
        b.mass[i] = a.mass[src];
        b.id[i] = a.id[src];
    }
    /* collide (particles_kernel.cuh:459-549): 3x3 cells, y outer, x inner,
     * per-cell subtotal */
    std::vector<V2<B>> acc(n);
    std::vector<T<B>> alpha(n);
    for (uint32_t i = 0; i < n; ++i) {
        const V2<B> p = b.pos[i], v = b.vel[i];
        const T<B> w = b.omega[i];
        const B r = b.radius[i];
        int gx, gy;
        grid_pos(s, p.x.v, p.y.v, &gx, &gy);
        V2<B> force = v2(T<B>(0), T<B>(0));
        T<B> moment(0);
        for (int y = -1; y <= 1; ++y) {
            for (int x = -1; x <= 1; ++x) {
                const uint32_t h = grid_hash(s, gx + x, gy + y);
                const uint32_t st = cellStart[h];
                V2<B> fc = v2(T<B>(0), T<B>(0));
                if (st != 0xffffffffu) {
                    for (uint32_t j = st; j < cellEnd[h]; ++j) {
                        if (j == i) continue;
                        const V2<B> f = collide_spheres(s, p, b.pos[j], v, b.vel[j], w,
                                                        b.omega[j], r, b.radius[j], moment);
                        fc.x = fc.x + f.x;
                        fc.y = fc.y + f.y;
                    }
                }
                force.x = force.x + fc.x;
                force.y = force.y + fc.y;
            }
        }
        const B m = b.mass[i];
        acc[i] = v2(force.x / T<B>(m), force.y / T<B>(m));
        alpha[i] = moment / inertia(m, r);
    }
    /* integrate (particles_kernel.cuh:580-627) */
    const double twopi = 2 * M_PI;
    const T<B> dt(s.dt);
    for (uint32_t i = 0; i < n; ++i) {
        V2<B> p = b.pos[i], v = b.vel[i];
        const V2<B> ac = acc[i];
        v.x = v.x + (T<B>(s.gravx) + ac.x) * dt;
        v.y = v.y + (T<B>(s.gravy) + ac.y) * dt;
        p.x = p.x + v.x * dt;
        p.y = p.y + v.y * dt;
        T<B> w = b.omega[i] + alpha[i] * dt;
        B th = b.theta[i] + w.v * s.dt;
        if (th > twopi) th = (B)((double)th - twopi * std::floor((double)th / twopi));
        if (th < 0) th = (B)((double)th - twopi * std::floor((double)th / twopi));
        const B r = b.radius[i];
        const T<B> eb(-s.m.eb);
        uint64_t wb = 0;
        if (p.x.v > s.Lx - r) { p.x = T<B>(s.Lx - r); v.x = v.x * eb; wb |= 1u; }
        if (p.x.v < r) { p.x = T<B>(r); v.x = v.x * eb; wb |= 2u; }
        if (p.y.v > s.Ly - r) { p.y = T<B>(s.Ly - r); v.y = v.y * eb; wb |= 4u; }
        if (wb) sig_mix(0x100u | wb);
        if (p.y.v < r) {
            sig_mix(0x200u | ((uint64_t)i << 12));
            T<B> wa(0);
            const V2<B> aw = collide_floor(s, p, v, w, r, b.mass[i], wa);
            v.x = v.x + aw.x * dt;
            v.y = v.y + aw.y * dt;
            p.x = p.x + aw.x * dt * dt;
            p.y = p.y + aw.y * dt * dt;
            w = w + wa * dt;
            th += wa.v * s.dt * s.dt;
            p.y = T<B>(r);
            v.y = v.y * eb;
        }
        b.pos[i] = p;
        b.vel[i] = v;
        b.omega[i] = w;
        b.theta[i] = th;
    }
    *sig = g_sig;
}

template <typename B>
T<B> seeded(double v, const double* d, size_t stride) {
    T<B> r((B)v);
    for (int k = 0; k < K; ++k) r.d[k] = (B)d[k * stride];
    return r;
}

template <typename B>
int run(const OrcSystem* os, uint32_t n, uint32_t steps, double* pos, double* vel,
        double* theta, double* omega, double* radius, double* mass, uint32_t* id,
        const double* dmat, const double* dwall, double* dpos, double* dvel, double* domega,
        uint64_t* signature) {
    if (os->nmat != 1 || os->mat[0][5] != 0.0) return -1;
    Sys<B> s;
    s.Lx = (B)os->Lx; s.Ly = (B)os->Ly; s.dt = (B)os->dt;
    s.gx = os->gx; s.gy = os->gy;
    s.gx_f = (B)os->gx; s.gy_f = (B)os->gy;
    s.gravx = (B)os->gravx; s.gravy = (B)os->gravy;
    /* dmat: [K][6] tangents of (kn, kt, cn, eb, mu, at); dwall: [K][2] of (knWall, ktWall) */
    s.m.kn = seeded<B>(os->mat[0][0], dmat + 0, 6);
    s.m.kt = seeded<B>(os->mat[0][1], dmat + 1, 6);
    s.m.cn = seeded<B>(os->mat[0][2], dmat + 2, 6);
    s.m.eb = (B)os->mat[0][3];
    s.m.mu = seeded<B>(os->mat[0][4], dmat + 4, 6);
    s.ktWall = seeded<B>(os->ktWall, dwall + 1, 2);
    State<B> a, b;
    for (State<B>* st : {&a, &b}) {
        st->pos.resize(n); st->vel.resize(n); st->omega.resize(n);
        st->theta.resize(n); st->radius.resize(n); st->mass.resize(n); st->id.resize(n);
    }
    const size_t n2 = 2ull * n;
    for (uint32_t i = 0; i < n; ++i) {
        a.pos[i] = v2(seeded<B>(pos[2 * i], dpos + 2 * i, n2), seeded<B>(pos[2 * i + 1], dpos + 2 * i + 1, n2));
        a.vel[i] = v2(seeded<B>(vel[2 * i], dvel + 2 * i, n2), seeded<B>(vel[2 * i + 1], dvel + 2 * i + 1, n2));
        a.omega[i] = seeded<B>(omega[i], domega + i, n);
        a.theta[i] = (B)theta[i];
        a.radius[i] = (B)radius[i];
        a.mass[i] = (B)mass[i];
        a.id[i] = id[i];
    }
    g_sig = 1469598103934665603ull;
    uint64_t sig = g_sig;
    for (uint32_t t = 0; t < steps; ++t) {
        step(s, a, b, &sig);
        std::swap(a, b);
    }
    for (uint32_t i = 0; i < n; ++i) {
        pos[2 * i] = a.pos[i].x.v; pos[2 * i + 1] = a.pos[i].y.v;
        vel[2 * i] = a.vel[i].x.v; vel[2 * i + 1] = a.vel[i].y.v;
        omega[i] = a.omega[i].v; theta[i] = a.theta[i];
        radius[i] = a.radius[i]; mass[i] = a.mass[i]; id[i] = a.id[i];
        for (int k = 0; k < K; ++k) {
            dpos[k * n2 + 2 * i] = a.pos[i].x.d[k];
            dpos[k * n2 + 2 * i + 1] = a.pos[i].y.d[k];
            dvel[k * n2 + 2 * i] = a.vel[i].x.d[k];
            dvel[k * n2 + 2 * i + 1] = a.vel[i].y.d[k];
            domega[k * (size_t)n + i] = a.omega[i].d[k];
        }
    }
    *signature = sig;
    return 0;
}

}  // namespace

/* Runs `steps` steps from the given state (arrays in and out; out = the
 * final sorted state) with K = 4 tangent directions.  Tangent arrays are
 * direction-major: dpos/dvel [4][n][2], domega [4][n] (in: initial tangents,
 * out: final), dmat [4][6], dwall [4][2].  Returns 0, or -1 for a system the
 * tangent does not cover (more than one material, or attraction). */
extern "C" int tan_run(const OrcSystem* os, uint32_t n, uint32_t steps, double* pos, double* vel,
                       double* theta, double* omega, double* radius, double* mass, uint32_t* id,
                       const double* dmat, const double* dwall, double* dpos, double* dvel,
                       double* domega, uint64_t* signature) {
#ifdef TAN_FLOAT
    return run<float>(os, n, steps, pos, vel, theta, omega, radius, mass, id, dmat, dwall, dpos,
                      dvel, domega, signature);
#else
    return run<double>(os, n, steps, pos, vel, theta, omega, radius, mass, id, dmat, dwall, dpos,
                       dvel, domega, signature);
#endif
}

extern "C" int tan_directions(void) { return K; }
