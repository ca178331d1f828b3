/* Test infrastructure (oracle only) -- never linked into the product.
 *
 * CPU restatement of the reference's per-timestep DEM step.  Each function
 * cites the reference lines it restates.  Compile with -DREAL=float or
 * -DREAL=double and -ffp-contract=off (no fused multiply-add), so the float
 * build performs exactly the IEEE operations the reference's source spells.
 *
 * Parity pin: the float build is checked bit-for-bit against the host build
 * of the reference's own kernels (oracle/_ref/libdemso_ref.so) by
 * tests/test_oracle.py and against tests/golden/ fixtures made from it.
 */
#include "dem_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#error "compile with -DREAL=float or -DREAL=double"
#endif

typedef struct { REAL x, y; } R2;

/* Branch signature: a running hash of every branch the contact law and the
 * integrator take (contact, dashpot, slip, walls, floor), so that a finite
 * difference whose +h and -h runs took different branches can be detected. */
static uint64_t g_sig = 1469598103934665603ull;
static inline void sig_mix(uint64_t v) { g_sig = (g_sig ^ v) * 1099511628211ull; }
void orc_signature_reset(void) { g_sig = 1469598103934665603ull; }
uint64_t orc_signature(void) { return g_sig; }

static inline R2 r2(REAL x, REAL y) { R2 v; v.x = x; v.y = y; return v; }
static inline R2 ld2(const REAL* a, uint32_t i) { return r2(a[2 * i], a[2 * i + 1]); }
static inline void st2(REAL* a, uint32_t i, R2 v) { a[2 * i] = v.x; a[2 * i + 1] = v.y; }
static inline REAL dot2(R2 a, R2 b) { return a.x * b.x + a.y * b.y; }
static inline REAL len2(R2 a) {
    REAL d = dot2(a, a);
    return (sizeof(REAL) == sizeof(float)) ? (REAL)sqrtf((float)d) : (REAL)sqrt((double)d);
}
static inline REAL rfloor(REAL v) {
    return (sizeof(REAL) == sizeof(float)) ? (REAL)floorf((float)v) : (REAL)floor((double)v);
}

/* particles_kernel.cuh:36-41 */
static inline REAL series(REAL a, REAL b) {
    if (a == 0.0 || b == 0.0) return 0.0;
    return (a * b) / (a + b);
}

typedef struct {
    REAL Lx, Ly, dt, gx_f, gy_f, gravx, gravy, knWall, ktWall;
    uint32_t gx, gy;
    REAL kn[ORC_MAX_MATERIALS], kt[ORC_MAX_MATERIALS], cn[ORC_MAX_MATERIALS];
    REAL eb[ORC_MAX_MATERIALS], mu[ORC_MAX_MATERIALS], at[ORC_MAX_MATERIALS];
} Sys;

static Sys load_sys(const OrcSystem* s) {
    Sys o;
    o.Lx = (REAL)s->Lx; o.Ly = (REAL)s->Ly; o.dt = (REAL)s->dt;
    o.gx = s->gx; o.gy = s->gy;
    o.gx_f = (REAL)s->gx; o.gy_f = (REAL)s->gy;
    o.gravx = (REAL)s->gravx; o.gravy = (REAL)s->gravy;
    o.knWall = (REAL)s->knWall; o.ktWall = (REAL)s->ktWall;
    for (int m = 0; m < ORC_MAX_MATERIALS; ++m) {
        o.kn[m] = (REAL)s->mat[m][0]; o.kt[m] = (REAL)s->mat[m][1];
        o.cn[m] = (REAL)s->mat[m][2]; o.eb[m] = (REAL)s->mat[m][3];
        o.mu[m] = (REAL)s->mat[m][4]; o.at[m] = (REAL)s->mat[m][5];
    }
    return o;
}

static inline uint32_t mat_of(const uint32_t* type, uint32_t i) { return type ? type[i] : 0u; }

/* main.cu:193 -- inertia 2/5 m r^2, evaluated left to right */
static inline REAL inertia_of(REAL m, REAL r) { return 2 * m * r * r / 5; }

/* particles_kernel.cuh:114-121 (float multiply, then IEEE divide, floor) */
static inline void grid_pos(const Sys* s, R2 p, int* gx, int* gy) {
    *gx = (int)rfloor(p.x * s->gx_f / s->Lx);
    *gy = (int)rfloor(p.y * s->gy_f / s->Ly);
}

/* particles_kernel.cuh:124-130 (power-of-two wrap) */
static inline uint32_t grid_hash(const Sys* s, int x, int y) {
    x = x & (int)(s->gx - 1);
    y = y & (int)(s->gy - 1);
    return (uint32_t)y * s->gx + (uint32_t)x;
}

/* particles_kernel.cuh:133-151 */
void orc_calc_hash(const OrcSystem* os, uint32_t n, const REAL* pos, uint32_t* hash,
                   uint32_t* index) {
    Sys s = load_sys(os);
    for (uint32_t i = 0; i < n; ++i) {
        int x, y;
        grid_pos(&s, ld2(pos, i), &x, &y);
        hash[i] = grid_hash(&s, x, y);
        index[i] = i;
    }
}

/* functions.cu:336-341: sort_by_key is a stable ascending radix sort.
 * Restated as a stable LSD radix sort, 8 bits per pass. */
void orc_sort(uint32_t n, uint32_t* hash, uint32_t* index) {
    uint32_t* k2 = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t* v2 = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *ks = hash, *vs = index, *kd = k2, *vd = v2;
    for (int shift = 0; shift < 32; shift += 8) {
        uint32_t cnt[257];
        memset(cnt, 0, sizeof(cnt));
        for (uint32_t i = 0; i < n; ++i) cnt[((ks[i] >> shift) & 255u) + 1]++;
        for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t d = (ks[i] >> shift) & 255u;
            uint32_t o = cnt[d]++;
            kd[o] = ks[i];
            vd[o] = vs[i];
        }
        uint32_t* t = ks; ks = kd; kd = t;
        t = vs; vs = vd; vd = t;
    }
    /* four passes: the result is back in hash/index */
    free(k2);
    free(v2);
}

/* functions.cu:371 (cellStart <- 0xFFFFFFFF) and particles_kernel.cuh:156-233.
 * cellEnd is not reset, as in the reference. */
void orc_reorder(const OrcSystem* os, uint32_t n, uint32_t* cellStart, uint32_t* cellEnd,
                 REAL* sPos, REAL* sVel, REAL* sTheta, REAL* sOmega, REAL* sRadius, REAL* sMass,
                 uint32_t* sID, uint32_t* sLoc, uint32_t* sType,
                 const uint32_t* hash, const uint32_t* index,
                 const REAL* oPos, const REAL* oVel, const REAL* oTheta, const REAL* oOmega,
                 const REAL* oRadius, const REAL* oMass, const uint32_t* oID,
                 const uint32_t* oType) {
    memset(cellStart, 0xff, sizeof(uint32_t) * (size_t)os->gx * os->gy);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t h = hash[i];
        if (i == 0 || h != hash[i - 1]) {
            cellStart[h] = i;
            if (i > 0) cellEnd[hash[i - 1]] = i;
        }
        if (i == n - 1) cellEnd[h] = i + 1;
        uint32_t src = index[i];
        st2(sPos, i, ld2(oPos, src));
        st2(sVel, i, ld2(oVel, src));
        sTheta[i] = oTheta[src];
        sOmega[i] = oOmega[src];
        sRadius[i] = oRadius[src];
        sMass[i] = oMass[src];
        sID[i] = oID[src];
        sLoc[oID[src]] = i;
        if (sType) sType[i] = oType[src];
    }
}

/* particles_kernel.cuh:236-307 (collideSpheres) */
static R2 collide_spheres(const Sys* s, R2 pA, R2 pB, R2 vA, R2 vB, REAL wA, REAL wB,
                          REAL rA, REAL rB, uint32_t mA, uint32_t mB, REAL* moment,
                          float* pressure) {
    R2 rel = r2(pB.x - pA.x, pB.y - pA.y);
    REAL dist = len2(rel);
    REAL cd = rA + rB;
    R2 force = r2(0, 0);
    if (dist < cd) {
        R2 nrm = r2(rel.x / dist, rel.y / dist);
        R2 tng = r2(-nrm.y, nrm.x);
        R2 rv = r2(vB.x - vA.x, vB.y - vA.y);
        REAL vn = dot2(rv, nrm);
        R2 vt = r2(rv.x - vn * nrm.x, rv.y - vn * nrm.y);
        REAL kn = series(s->kn[mA], s->kn[mB]);
        REAL kt = series(s->kt[mA], s->kt[mB]);
        REAL cn = series(s->cn[mA], s->cn[mB]);
        REAL mu = (s->mu[mA] + s->mu[mB]) / 2;
        REAL fs = -kn * (cd - dist);
        force = r2(fs * nrm.x, fs * nrm.y);
        if (vn < 0) {
            REAL c = cn * vn;
            force.x += c * nrm.x;
            force.y += c * nrm.y;
        }
        *pressure = (float)((double)*pressure + (double)len2(force) / (4 * M_PI * rA * rA));
        uint64_t br = 1u | (vn < 0 ? 2u : 0u);
        if (mu != 0.0) {
            REAL sw = rA * wA + rB * wB;
            R2 vc = r2(vt.x - sw * tng.x, vt.y - sw * tng.y);
            R2 ftr = r2(kt * vc.x * s->dt, kt * vc.y * s->dt);
            REAL ftmax = mu * len2(force);
            R2 ft;
            if (len2(ftr) < ftmax) {
                ft = ftr;
            } else {
                REAL l = len2(vc);
                ft = r2(ftmax * vc.x / l, ftmax * vc.y / l);
                br |= 4u;
            }
            force.x += ft.x;
            force.y += ft.y;
            *moment += rA * dot2(ft, tng);
        }
        sig_mix(br);
    }
    return force;
}

/* particles_kernel.cuh:311-342 (attractSpheres) */
static R2 attract_spheres(const Sys* s, R2 pA, R2 pB, REAL rA, REAL rB, uint32_t mA,
                          uint32_t mB, float* pressure) {
    R2 rel = r2(pB.x - pA.x, pB.y - pA.y);
    REAL dist = len2(rel);
    /* `radius * 2 * 1.2`: float product, then a double multiply by 1.2 */
    REAL dA = (REAL)((double)(rA * 2) * 1.2);
    REAL dB = (REAL)((double)(rB * 2) * 1.2);
    R2 nrm = r2(rel.x / dist, rel.y / dist);
    R2 force = r2(0, 0);
    if (dist < dA) {
        REAL c = s->at[mA] * (dA - dist);
        force.x += c * nrm.x;
        force.y += c * nrm.y;
    }
    if (dist < dB) {
        REAL c = s->at[mB] * (dB - dist);
        force.x += c * nrm.x;
        force.y += c * nrm.y;
    }
    *pressure = (float)((double)*pressure + (double)len2(force) / (4 * M_PI * rA * rA));
    return force;
}

/* functions.cu:441 (pressure <- 0) and particles_kernel.cuh:459-549 with
 * USE_BIG_PARTICLE 0: 3x3 neighbour cells, y outer, x inner; each cell's
 * subtotal (collideCell, :346-385) is added to the running force. */
static void collide_impl(const OrcSystem* os, uint32_t n, const REAL* pos, const REAL* vel,
                         const REAL* omega, const REAL* radius, const REAL* mass,
                         const uint32_t* type, const uint32_t* cellStart, const uint32_t* cellEnd,
                         REAL* acc, REAL* alpha, float* pressure, const OrcControl* ctl,
                         REAL* fx, REAL* fy, REAL* fm);

void orc_collide(const OrcSystem* os, uint32_t n, const REAL* pos, const REAL* vel,
                 const REAL* omega, const REAL* radius, const REAL* mass, const uint32_t* type,
                 const uint32_t* cellStart, const uint32_t* cellEnd, REAL* acc, REAL* alpha,
                 float* pressure) {
    collide_impl(os, n, pos, vel, omega, radius, mass, type, cellStart, cellEnd, acc, alpha,
                 pressure, NULL, NULL, NULL, NULL);
}

/* particles_kernel.cuh:459-549 with USE_BIG_PARTICLE 1 and USE_ATOMIC 0: after
 * the 3x3 cells, the contact (and attraction) with the control particle is
 * added to the force and moment, and -f.x, -f.y and -m / rA * rControl are
 * stored per particle for the reduction. */
void orc_collide_control(const OrcSystem* os, uint32_t n, const REAL* pos, const REAL* vel,
                         const REAL* omega, const REAL* radius, const REAL* mass,
                         const uint32_t* type, const uint32_t* cellStart,
                         const uint32_t* cellEnd, REAL* acc, REAL* alpha, float* pressure,
                         const OrcControl* ctl, REAL* fx, REAL* fy, REAL* fm) {
    collide_impl(os, n, pos, vel, omega, radius, mass, type, cellStart, cellEnd, acc, alpha,
                 pressure, ctl, fx, fy, fm);
}

static void collide_impl(const OrcSystem* os, uint32_t n, const REAL* pos, const REAL* vel,
                         const REAL* omega, const REAL* radius, const REAL* mass,
                         const uint32_t* type, const uint32_t* cellStart, const uint32_t* cellEnd,
                         REAL* acc, REAL* alpha, float* pressure, const OrcControl* ctl,
                         REAL* fx, REAL* fy, REAL* fm) {
    Sys s = load_sys(os);
    for (uint32_t i = 0; i < n; ++i) {
        R2 p = ld2(pos, i), v = ld2(vel, i);
        REAL w = omega[i], r = radius[i];
        uint32_t mi = mat_of(type, i);
        int gx, gy;
        grid_pos(&s, p, &gx, &gy);
        R2 force = r2(0, 0);
        REAL moment = 0;
        float pr = 0.0f;
        for (int y = -1; y <= 1; ++y) {
            for (int x = -1; x <= 1; ++x) {
                uint32_t h = grid_hash(&s, gx + x, gy + y);
                uint32_t st = cellStart[h];
                R2 fc = r2(0, 0);
                if (st != 0xffffffffu) {
                    uint32_t en = cellEnd[h];
                    for (uint32_t j = st; j < en; ++j) {
                        if (j == i) continue;
                        uint32_t mj = mat_of(type, j);
                        R2 f = collide_spheres(&s, p, ld2(pos, j), v, ld2(vel, j), w, omega[j],
                                               r, radius[j], mi, mj, &moment, &pr);
                        fc.x += f.x; fc.y += f.y;
                        f = attract_spheres(&s, p, ld2(pos, j), r, radius[j], mi, mj, &pr);
                        fc.x += f.x; fc.y += f.y;
                    }
                }
                force.x += fc.x;
                force.y += fc.y;
            }
        }
        if (ctl) {
            REAL mc = 0;
            const R2 cp = r2((REAL)ctl->pos[0], (REAL)ctl->pos[1]);
            const REAL cr = (REAL)ctl->radius;
            R2 f = collide_spheres(&s, p, cp, v, r2((REAL)ctl->vel[0], (REAL)ctl->vel[1]), w,
                                   (REAL)ctl->omega, r, cr, mi, ctl->mat, &mc, &pr);
            const R2 fa = attract_spheres(&s, p, cp, r, cr, mi, ctl->mat, &pr);
            f.x += fa.x;
            f.y += fa.y;
            force.x += f.x;
            force.y += f.y;
            moment += mc;
            fx[i] = -f.x;
            fy[i] = -f.y;
            fm[i] = -mc / r * cr;
        }
        REAL m = mass[i];
        st2(acc, i, r2(force.x / m, force.y / m));
        alpha[i] = moment / inertia_of(m, r);
        pressure[i] = pr;
    }
}

/* particles_kernel.cuh:388-456 (collideBoundary) against the floor point (x, 0) */
static R2 collide_floor(const Sys* s, R2 p, R2 v, REAL w, REAL r, REAL m, uint32_t mi,
                        REAL* walpha, float* pressure) {
    R2 rel = r2(p.x - p.x, (REAL)0 - p.y);
    REAL dist = len2(rel);
    R2 force = r2(0, 0);
    if (dist < r) {
        R2 nrm = r2(rel.x / dist, rel.y / dist);
        R2 tng = r2(-nrm.y, nrm.x);
        R2 rv = r2(-v.x, -v.y);
        REAL vn = dot2(rv, nrm);
        R2 vt = r2(rv.x - vn * nrm.x, rv.y - vn * nrm.y);
        REAL kt = series(s->kt[mi], s->ktWall);
        REAL cn = s->cn[mi];
        REAL nm = -m;
        force = r2(nm * s->gravx, nm * s->gravy);
        if (vn < 0) {
            REAL c = cn * vn;
            force.x += c * nrm.x;
            force.y += c * nrm.y;
        }
        *pressure = (float)((double)*pressure + (double)len2(force) / (4 * M_PI * r * r));
        if (s->mu[mi] != 0.0) {
            REAL rw = r * w;
            R2 vc = r2(vt.x - rw * tng.x, vt.y - rw * tng.y);
            R2 ftr = r2(kt * vc.x * s->dt, kt * vc.y * s->dt);
            REAL ftmax = s->mu[mi] * len2(force);
            R2 ft;
            if (len2(ftr) < ftmax) {
                ft = ftr;
            } else {
                REAL l = len2(vc);
                ft = r2(ftmax * vc.x / l, ftmax * vc.y / l);
            }
            force = ft;
            *walpha += r * dot2(ft, tng) / inertia_of(m, r);
        }
    }
    return r2(force.x / m, force.y / m);
}

/* particles_kernel.cuh:580-627 (integrateSystemD) */
void orc_integrate(const OrcSystem* os, uint32_t n, REAL* pos, REAL* vel, const REAL* acc,
                   REAL* theta, REAL* omega, const REAL* alpha, const REAL* radius,
                   const REAL* mass, const uint32_t* type, float* pressure) {
    Sys s = load_sys(os);
    const double twopi = 2 * M_PI;
    for (uint32_t i = 0; i < n; ++i) {
        R2 p = ld2(pos, i), v = ld2(vel, i), a = ld2(acc, i);
        v.x += (s.gravx + a.x) * s.dt;
        v.y += (s.gravy + a.y) * s.dt;
        p.x += v.x * s.dt;
        p.y += v.y * s.dt;
        REAL w = omega[i] + alpha[i] * s.dt;
        REAL th = theta[i] + w * s.dt;
        if (th > twopi) th = (REAL)((double)th - twopi * floor((double)th / twopi));
        if (th < 0) th = (REAL)((double)th - twopi * floor((double)th / twopi));
        REAL r = radius[i];
        uint32_t mi = mat_of(type, i);
        REAL eb = s.eb[mi];
        uint64_t wb = 0;
        if (p.x > s.Lx - r) { p.x = s.Lx - r; v.x *= -eb; wb |= 1u; }
        if (p.x < r) { p.x = r; v.x *= -eb; wb |= 2u; }
        if (p.y > s.Ly - r) { p.y = s.Ly - r; v.y *= -eb; wb |= 4u; }
        if (wb) sig_mix(0x100u | wb);
        if (p.y < r) {
            sig_mix(0x200u | ((uint64_t)i << 12));
            REAL wa = 0;
            R2 aw = collide_floor(&s, p, v, w, r, mass[i], mi, &wa, &pressure[i]);
            v.x += aw.x * s.dt;
            v.y += aw.y * s.dt;
            p.x += aw.x * s.dt * s.dt;
            p.y += aw.y * s.dt * s.dt;
            w += wa * s.dt;
            th += wa * s.dt * s.dt;
            p.y = r;
            v.y *= -eb;
        }
        st2(pos, i, p);
        st2(vel, i, v);
        omega[i] = w;
        theta[i] = th;
    }
}

/* One full step in the order of SimLooping (main.cu:431-507), from state
 * buffer set A into set B (B is the sorted, integrated state on return).
 * Scratch: acc[2n], alpha[n], pressure[n], hash[n], index[n], cellStart/End. */
void orc_step(const OrcSystem* os, uint32_t n,
              const REAL* aPos, const REAL* aVel, const REAL* aTheta, const REAL* aOmega,
              const REAL* aRadius, const REAL* aMass, const uint32_t* aID, const uint32_t* aType,
              REAL* bPos, REAL* bVel, REAL* bTheta, REAL* bOmega, REAL* bRadius, REAL* bMass,
              uint32_t* bID, uint32_t* bLoc, uint32_t* bType,
              REAL* acc, REAL* alpha, float* pressure, uint32_t* hash, uint32_t* index,
              uint32_t* cellStart, uint32_t* cellEnd) {
    orc_calc_hash(os, n, aPos, hash, index);
    orc_sort(n, hash, index);
    orc_reorder(os, n, cellStart, cellEnd, bPos, bVel, bTheta, bOmega, bRadius, bMass, bID, bLoc,
                aType ? bType : NULL, hash, index, aPos, aVel, aTheta, aOmega, aRadius, aMass,
                aID, aType);
    orc_collide(os, n, bPos, bVel, bOmega, bRadius, bMass, aType ? bType : NULL, cellStart,
                cellEnd, acc, alpha, pressure);
    orc_integrate(os, n, bPos, bVel, acc, bTheta, bOmega, alpha, bRadius, bMass,
                  aType ? bType : NULL, pressure);
}

int orc_real_bytes(void) { return (int)sizeof(REAL); }

/* reduceVecD (particles_kernel.cuh:551-578) over blocks of
 * min(512, n) entries as collide launches it (functions.cu:486-488), then the
 * host's sum of the block results in block order (functions.cu:511-519), in
 * float. */
float orc_control_reduce(uint32_t n, const float* v) {
    if (n == 0) return 0.0f;
    const uint32_t threads = n < 512u ? n : 512u;
    const uint32_t blocks = (n % threads != 0) ? n / threads + 1 : n / threads;
    float* cache = (float*)malloc(sizeof(float) * threads);
    float sum = 0.0f;
    for (uint32_t b = 0; b < blocks; ++b) {
        for (uint32_t t = 0; t < threads; ++t) {
            const uint32_t idx = b * threads + t;
            cache[t] = idx < n ? v[idx] : 0.0f;
        }
        for (uint32_t i = threads / 2; i != 0; i /= 2)
            for (uint32_t t = 0; t < i; ++t) cache[t] += cache[t + i];
        sum += cache[0];
    }
    free(cache);
    return sum;
}

/* main.cu:511-514: the host moves the control particle after each step, in
 * double rounded to float as `float += double` does. */
void orc_control_move(OrcControl* c) {
    c->pos[0] = (float)((double)(float)c->pos[0] + c->drift[0]);
    c->pos[1] = (float)((double)(float)c->pos[1] + c->drift[1]);
    if (c->wrapYBelow == c->wrapYBelow && (float)c->pos[1] < c->wrapYBelow)
        c->pos[1] = (float)c->wrapYTo;
    if (c->wrapXAbove == c->wrapXAbove && (double)(float)c->pos[0] > c->wrapXAbove)
        c->pos[0] = (float)c->wrapXTo;
}
