/* Test infrastructure (oracle only) -- never linked into the product.
 *
 * CPU restatement of DemSo's per-timestep DEM step, written from the
 * reference's algorithm (src/particles_kernel.cuh, src/functions.cu,
 * src/main.cu).  dem_oracle.c is compiled twice: with REAL = float
 * (libdem_oracle_f32.so, no FP contraction, pinned bit-exact against the
 * host build of the reference's own kernels in oracle/_ref) and with
 * REAL = double (libdem_oracle_f64.so, the FP64 trajectory oracle).
 *
 * Layout is the reference's: pos/vel/acc are float2 arrays passed as REAL*
 * with 2 entries per particle, everything else one entry per particle.
 * Per-particle radius and mass replace the reference's per-type table; the
 * contact coefficients come from a small material table indexed by
 * `type` (NULL = material 0 for every particle).
 */
#ifndef DEMSO_ORACLE_H
#define DEMSO_ORACLE_H
#include <stdint.h>

#define ORC_MAX_MATERIALS 10

typedef struct OrcSystem {
    double Lx, Ly;           /* cubeDimension (main.cuh:112) */
    uint32_t gx, gy;         /* gridSize, powers of two (main.cuh:113) */
    double dt;               /* timeStep */
    double gravx, gravy;     /* gravity */
    double knWall, ktWall;   /* boundaryNormalStiffness / boundaryShearStiffness */
    uint32_t nmat, reserved;
    /* per material: normalStiffness, shearStiffness, normalDamping,
     * boundaryDamping, frictionCoefficient, attractCoefficient */
    double mat[ORC_MAX_MATERIALS][6];
} OrcSystem;

/* The control ("big") particle of the reference built with
 * USE_BIG_PARTICLE 1: a kinematic disk of material `mat` touching every
 * particle (particles_kernel.cuh:520-541), moved by the host after each step
 * (main.cu:511-514 with drift (0, -0.005), wrapY (-1 -> 10.5) and wrapX
 * (Lx + 0.5 -> -0.5)).  A wrap is off when its threshold is NaN. */
typedef struct OrcControl {
    double pos[2], vel[2];
    double theta, omega, radius;
    uint32_t mat, reserved;
    double drift[2];
    double wrapYBelow, wrapYTo, wrapXAbove, wrapXTo;
} OrcControl;

#endif
