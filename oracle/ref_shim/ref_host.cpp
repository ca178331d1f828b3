/* Test infrastructure (oracle only) -- never linked into the product.
 *
 * Host build of the reference's OWN device code.  The reference header
 * src/particles_kernel.cuh is included unmodified from the reference tree
 * (path supplied by oracle/Makefile with -I); this file only supplies what
 * the header expects from its surroundings and drives its __global__
 * functions one "CUDA thread" at a time on host cores:
 *
 *  - the CUDA qualifiers become plain C++ (__shared__ becomes thread_local so
 *    each OpenMP thread has its own copy of the shared-memory scratch);
 *  - threadIdx/blockIdx/blockDim/gridDim are thread_local, with blockDim = 1,
 *    so the block-level handshake in reorderDataAndFindCellStartD
 *    (particles_kernel.cuh:175-195) is exact: thread 0 of every one-thread
 *    block loads hash[index-1] itself;
 *  - MAIN_CUH is pre-defined so the reference's main.cuh is skipped and the
 *    structs below are used instead.  They carry the field names the kernel
 *    header reads (main.cuh:39-135) with USE_BIG_PARTICLE = 0 (no control
 *    particle) and MAX_PARTICLES_TYPES large enough that every particle is its
 *    own "type", which gives per-particle radius, mass and inertia;
 *  - thrust::sort_by_key (functions.cu:336-341, a stable LSD radix sort) is
 *    replaced by std::stable_sort on (hash, index), the same order.
 *
 * The memsets the reference's host wrappers issue (functions.cu:371 and :441)
 * are reproduced in the stage functions below.
 */
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <utility>
#ifdef _OPENMP
#include <omp.h>
#endif

#undef __shared__
#define __shared__ thread_local

typedef unsigned int uint;

#define MAIN_CUH 1
#ifdef REF_CONTROL
#define USE_BIG_PARTICLE 1  /* with the control particle, USE_ATOMIC 0 (main.cuh:29-30) */
#else
#define USE_BIG_PARTICLE 0
#endif
#define USE_ATOMIC 0
#define MAX_PARTICLES_TYPES (1u << 24)

struct ParticleProperties {
    float radius, mass, inertia;
    float normalStiffness, shearStiffness, normalDamping, boundaryDamping;
    float frictionCoefficient, attractCoefficient;
    float colorR, colorG, colorB;
};

struct SystemProperties {
    uint numParticles;
    float2 cubeDimension;
    uint2 gridSize;
    uint numCells;
    float timeStep;
    float2 gravity;
    float boundaryNormalStiffness;
    float boundaryShearStiffness;
};

struct RenderParameters {
    int imageDIMx, imageDIMy, dimx, dimy;
    float pRadius;
    int bgColor;
    bool viewRotations, colorByPressure;
    float maxPressure;
};

static thread_local uint3 threadIdx;
static thread_local uint3 blockIdx;
static thread_local dim3 blockDim;
static thread_local dim3 gridDim;
static inline void __syncthreads() {}

/* per-thread storage for the header's `extern __shared__` scratch arrays */
thread_local uint sharedHash[2];
thread_local float cache[1];

#include "particles_kernel.cuh"

namespace {

inline void set_thread(uint i, uint n) {
    threadIdx = make_uint3(0, 0, 0);
    blockIdx = make_uint3(i, 0, 0);
    blockDim = dim3(1, 1, 1);
    gridDim = dim3(n, 1, 1);
}

}  // namespace

extern "C" {

/* Material row layout: kn, kt, cn, boundaryDamping, friction, attraction. */
int ref_max_particles(void) { return (int)MAX_PARTICLES_TYPES; }

int ref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

/* Fill the constant-memory stand-ins.  Particle i becomes type i with the
 * radius/mass given and the contact coefficients of material[i]; inertia is
 * computed as main.cu:193 does. */
int ref_setup(uint32_t n, float Lx, float Ly, uint32_t gx, uint32_t gy, float dt,
              float gravx, float gravy, float knWall, float ktWall,
              const float* radius, const float* mass, const uint32_t* material,
              const float* matTable, uint32_t nmat) {
    if (n > MAX_PARTICLES_TYPES) return 1;
    sisPropD.numParticles = n;
    sisPropD.cubeDimension = make_float2(Lx, Ly);
    sisPropD.gridSize = make_uint2(gx, gy);
    sisPropD.numCells = gx * gy;
    sisPropD.timeStep = dt;
    sisPropD.gravity = make_float2(gravx, gravy);
    sisPropD.boundaryNormalStiffness = knWall;
    sisPropD.boundaryShearStiffness = ktWall;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t m = material ? material[i] : 0u;
        if (m >= nmat) return 2;
        const float* row = matTable + 6 * m;
        ParticleProperties& p = partPropD[i];
        p.radius = radius[i];
        p.mass = mass[i];
        p.inertia = 2 * p.mass * p.radius * p.radius / 5;
        p.normalStiffness = row[0];
        p.shearStiffness = row[1];
        p.normalDamping = row[2];
        p.boundaryDamping = row[3];
        p.frictionCoefficient = row[4];
        p.attractCoefficient = row[5];
        p.colorR = p.colorG = p.colorB = 255.0f;
    }
    return 0;
}

void ref_set_gravity(float gravx, float gravy) { sisPropD.gravity = make_float2(gravx, gravy); }

void ref_calc_hash(const float* pos, uint32_t* hash, uint32_t* index) {
    const uint n = sisPropD.numParticles;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; ++i) {
        set_thread((uint)i, n);
        calcHashD(hash, index, (float2*)pos);
    }
}

void ref_sort(uint32_t* hash, uint32_t* index) {
    const uint n = sisPropD.numParticles;
    std::vector<std::pair<uint32_t, uint32_t>> kv(n);
    for (uint i = 0; i < n; ++i) kv[i] = std::make_pair(hash[i], index[i]);
    std::stable_sort(kv.begin(), kv.end(),
                     [](const std::pair<uint32_t, uint32_t>& a,
                        const std::pair<uint32_t, uint32_t>& b) { return a.first < b.first; });
    for (uint i = 0; i < n; ++i) { hash[i] = kv[i].first; index[i] = kv[i].second; }
}

void ref_reorder(uint32_t* cellStart, uint32_t* cellEnd,
                 float* sortedPos, float* sortedVel, float* sortedTheta, float* sortedOmega,
                 uint32_t* sortedID, uint32_t* sortedLoc, uint32_t* sortedType,
                 uint32_t* hash, uint32_t* index,
                 float* oldPos, float* oldVel, float* oldTheta, float* oldOmega,
                 uint32_t* oldID, uint32_t* oldType) {
    const uint n = sisPropD.numParticles;
    memset(cellStart, 0xff, sizeof(uint32_t) * sisPropD.numCells);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; ++i) {
        set_thread((uint)i, n);
        reorderDataAndFindCellStartD(cellStart, cellEnd, (float2*)sortedPos, (float2*)sortedVel,
                                     sortedTheta, sortedOmega, sortedID, sortedLoc, sortedType,
                                     hash, index, (float2*)oldPos, (float2*)oldVel, oldTheta,
                                     oldOmega, oldID, oldType);
    }
}

#if USE_BIG_PARTICLE
/* The control particle (main.cu:141-146, 476-494): its kinematic state and
 * the per-particle reaction vectors collideD writes (USE_ATOMIC 0). */
static float2 g_cPos, g_cVel;
static float g_cTheta, g_cOmega;
static uint g_cType;
static std::vector<float> g_fx, g_fy, g_fm;

/* Call after ref_setup: the control particle becomes type n (one past the
 * particles) with the given radius, mass and material row. */
int ref_set_control(float px, float py, float vx, float vy, float theta, float omega,
                    float radius, float mass, const float* row) {
    const uint n = sisPropD.numParticles;
    if (n + 1 > MAX_PARTICLES_TYPES) return 1;
    ParticleProperties& p = partPropD[n];
    p.radius = radius;
    p.mass = mass;
    p.inertia = 2 * p.mass * p.radius * p.radius / 5;
    p.normalStiffness = row[0];
    p.shearStiffness = row[1];
    p.normalDamping = row[2];
    p.boundaryDamping = row[3];
    p.frictionCoefficient = row[4];
    p.attractCoefficient = row[5];
    g_cPos = make_float2(px, py);
    g_cVel = make_float2(vx, vy);
    g_cTheta = theta;
    g_cOmega = omega;
    g_cType = n;
    return 0;
}

/* The reaction vectors of the last ref_collide (n entries each). */
void ref_control_vectors(float* fx, float* fy, float* fm) {
    const size_t n = g_fx.size();
    memcpy(fx, g_fx.data(), 4 * n);
    memcpy(fy, g_fy.data(), 4 * n);
    memcpy(fm, g_fm.data(), 4 * n);
}
#endif

void ref_collide(float* pos, float* vel, float* acc, float* omega, float* alpha, uint32_t* type,
                 uint32_t* cellStart, uint32_t* cellEnd, float* pressure) {
    const uint n = sisPropD.numParticles;
    memset(pressure, 0, sizeof(float) * n);
#if USE_BIG_PARTICLE
    g_fx.assign(n, 0.0f);
    g_fy.assign(n, 0.0f);
    g_fm.assign(n, 0.0f);
#endif
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; ++i) {
        set_thread((uint)i, n);
        collideD((float2*)pos, (float2*)vel, (float2*)acc, omega, alpha, type, cellStart,
                 cellEnd,
#if USE_BIG_PARTICLE
                 g_cPos, g_cVel, g_cTheta, g_cOmega, g_cType, g_fx.data(), g_fy.data(),
                 g_fm.data(),
#endif
                 pressure);
    }
}

void ref_integrate(float* pos, float* vel, float* acc, float* theta, float* omega, float* alpha,
                   uint32_t* type, float* pressure) {
    const uint n = sisPropD.numParticles;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; ++i) {
        set_thread((uint)i, n);
        integrateSystemD((float2*)pos, (float2*)vel, (float2*)acc, theta, omega, alpha, type,
                         pressure);
    }
}

/* `nsteps` full steps in the order of SimLooping (main.cu:396-507).  Buffer
 * set 1 holds the current state on entry and on return (an even number of
 * internal swaps is arranged by copying back when nsteps is odd).  Scratch
 * arrays are caller-provided so the timing covers only the step. */
void ref_run(uint32_t nsteps,
             float* pos1, float* vel1, float* theta1, float* omega1, uint32_t* id1,
             uint32_t* type1, uint32_t* loc1,
             float* pos2, float* vel2, float* theta2, float* omega2, uint32_t* id2,
             uint32_t* type2, uint32_t* loc2,
             float* acc, float* alpha, float* pressure, uint32_t* hash, uint32_t* index,
             uint32_t* cellStart, uint32_t* cellEnd) {
    const uint n = sisPropD.numParticles;
    for (uint32_t s = 0; s < nsteps; ++s) {
        const bool odd = (s & 1u) != 0;
        float* oP = odd ? pos2 : pos1;     float* sP = odd ? pos1 : pos2;
        float* oV = odd ? vel2 : vel1;     float* sV = odd ? vel1 : vel2;
        float* oT = odd ? theta2 : theta1; float* sT = odd ? theta1 : theta2;
        float* oW = odd ? omega2 : omega1; float* sW = odd ? omega1 : omega2;
        uint32_t* oI = odd ? id2 : id1;    uint32_t* sI = odd ? id1 : id2;
        uint32_t* oY = odd ? type2 : type1; uint32_t* sY = odd ? type1 : type2;
        uint32_t* sL = odd ? loc1 : loc2;
        ref_calc_hash(oP, hash, index);
        ref_sort(hash, index);
        ref_reorder(cellStart, cellEnd, sP, sV, sT, sW, sI, sL, sY, hash, index, oP, oV, oT, oW,
                    oI, oY);
        ref_collide(sP, sV, acc, sW, alpha, sY, cellStart, cellEnd, pressure);
        ref_integrate(sP, sV, acc, sT, sW, alpha, sY, pressure);
    }
    if (nsteps & 1u) {
        memcpy(pos1, pos2, sizeof(float) * 2 * n);
        memcpy(vel1, vel2, sizeof(float) * 2 * n);
        memcpy(theta1, theta2, sizeof(float) * n);
        memcpy(omega1, omega2, sizeof(float) * n);
        memcpy(id1, id2, sizeof(uint32_t) * n);
        memcpy(type1, type2, sizeof(uint32_t) * n);
        memcpy(loc1, loc2, sizeof(uint32_t) * n);
    }
}

/* The reference's disk splat, plotSpheresD (particles_kernel.cuh:656-734),
 * run one "CUDA thread" after the other in index order over the particles of
 * the last ref_setup (particle i is reference type i), with the rule the
 * library applies where the reference's threads race: a later particle's
 * disk covers an earlier one's, and the orientation lines come after every
 * disk.  `rgb` holds each particle's colour (3 floats), written into its
 * type's colorR/G/B; `pressure` may be NULL (zeros).  The image (dimx *
 * dimy RGBA bytes, row 0 at the bottom) is filled with bg first.
 *
 * The disks are one pass of calls with renderParD.viewRotations off.  The
 * pixels of particle i's line are found by calling the kernel for it again
 * twice over a scratch image filled with a sentinel, once with lines and
 * once without: a pixel the call with lines leaves all-zero and the call
 * without does not is a line pixel.  A pixel that the disk itself writes
 * all-zero (shade below 1/255) and that the line call also leaves all-zero
 * cannot be classed that way: such pixels are blackened and counted, and
 * the count is returned (and the pixels flagged in ambiguousMask, dimx * dimy
 * bytes, when it is not NULL).  Returns -1 when a particle's square reaches below
 * pixel 0 (the reference then converts negative floats to unsigned, which
 * the host does differently from the GPU). */
int ref_render(uint8_t* image, int dimx, int dimy, int bg, int viewRotations,
               int colorByPressure, float maxPressure, float* pos, float* theta,
               const float* rgb, float* pressure, uint8_t* ambiguousMask) {
    const uint n = sisPropD.numParticles;
    const size_t size = (size_t)dimx * dimy;
    renderParD.imageDIMx = dimx;
    renderParD.imageDIMy = dimy;
    renderParD.bgColor = bg;
    renderParD.colorByPressure = colorByPressure != 0;
    renderParD.maxPressure = maxPressure;
    std::vector<uint> type(n);
    std::vector<float> zeros;
    if (!pressure) {
        zeros.assign(n, 0.0f);
        pressure = zeros.data();
    }
    for (uint i = 0; i < n; ++i) {
        type[i] = i;
        partPropD[i].colorR = rgb[3 * i];
        partPropD[i].colorG = rgb[3 * i + 1];
        partPropD[i].colorB = rgb[3 * i + 2];
        const float pR = renderParD.imageDIMy / sisPropD.cubeDimension.y * partPropD[i].radius;
        const int cx = renderParD.imageDIMx / sisPropD.cubeDimension.x * pos[2 * i];
        const int cy = renderParD.imageDIMy / sisPropD.cubeDimension.y * pos[2 * i + 1];
        if (cx - (int)ceilf(pR) < 0 || cy - (int)ceilf(pR) < 0) return -1;
    }
    uchar4* img = reinterpret_cast<uchar4*>(image);
    const uchar4 bgc = make_uchar4(bg & 0xff, bg & 0xff, bg & 0xff, bg & 0xff);
    for (size_t p = 0; p < size; ++p) img[p] = bgc;
    renderParD.viewRotations = false;
    for (uint i = 0; i < n; ++i) {
        set_thread(i, n);
        plotSpheresD(img, reinterpret_cast<float2*>(pos), theta, type.data(), pressure);
    }
    if (!viewRotations) return 0;
    const uchar4 sentinel = make_uchar4(1, 2, 3, 4);
    std::vector<uchar4> on(size, sentinel), off(size, sentinel);
    std::vector<uint8_t> line(size, 0);
    auto zero = [](uchar4 c) { return c.x == 0 && c.y == 0 && c.z == 0 && c.w == 0; };
    int ambiguous = 0;
    for (uint i = 0; i < n; ++i) {
        const float pR = renderParD.imageDIMy / sisPropD.cubeDimension.y * partPropD[i].radius;
        const int cx = renderParD.imageDIMx / sisPropD.cubeDimension.x * pos[2 * i];
        const int cy = renderParD.imageDIMy / sisPropD.cubeDimension.y * pos[2 * i + 1];
        const int h = (int)ceilf(pR);
        // every pixel the call can write: its square, clamped to the last pixel
        std::vector<size_t> px;
        for (int y = cy - h; y < cy + h; ++y)
            for (int x = cx - h; x < cx + h; ++x) {
                size_t p = (size_t)(uint)x + (size_t)(uint)y * (uint)dimx;
                px.push_back(p < size ? p : size - 1);
            }
        px.push_back(size - 1);
        for (size_t p : px) on[p] = off[p] = sentinel;
        set_thread(i, n);
        renderParD.viewRotations = false;
        plotSpheresD(off.data(), reinterpret_cast<float2*>(pos), theta, type.data(), pressure);
        renderParD.viewRotations = true;
        plotSpheresD(on.data(), reinterpret_cast<float2*>(pos), theta, type.data(), pressure);
        for (size_t p : px) {
            if (line[p] || !zero(on[p])) continue;
            if (zero(off[p])) {
                ++ambiguous;
                if (ambiguousMask) ambiguousMask[p] = 1;
            }
            line[p] = 1;
        }
    }
    for (size_t p = 0; p < size; ++p)
        if (line[p]) img[p] = make_uchar4(0, 0, 0, 0);
    return ambiguous;
}

/* The reference's block generators, one "CUDA thread" per particle:
 * createRectanglesD (particles_kernel.cuh:43-74) with the cuRAND stand-in's
 * zero normal deviate, and createTrianglesD (:76-111) with space and height
 * formed as PrepareSim forms them (main.cu:306-307). */
void ref_create_rectangles(float* pos, uint32_t* id, uint32_t* loc, uint32_t* type, float sx,
                           float sy, float ex, float ey, uint32_t nx, uint32_t ny,
                           uint32_t startID, uint32_t ntypes, uint32_t* typeVec) {
    const float2 start = make_float2(sx, sy);
    const float2 len = make_float2(ex - sx, ey - sy);
    for (uint y = 0; y < ny; ++y)
        for (uint x = 0; x < nx; ++x) {
            threadIdx = make_uint3(0, 0, 0);
            blockIdx = make_uint3(x, y, 0);
            blockDim = dim3(1, 1, 1);
            gridDim = dim3(nx, ny, 1);
            createRectanglesD(reinterpret_cast<float2*>(pos), id, loc, type, start, len,
                              make_uint2(nx, ny), startID, ntypes, typeVec, 0ul);
        }
}

void ref_create_triangles(float* pos, uint32_t* id, uint32_t* loc, uint32_t* type, float px,
                          float py, float width, uint32_t N, uint32_t startID, uint32_t ntypes,
                          uint32_t* typeVec) {
    const uint32_t count = N * (N + 1) / 2;
    float space = width / (N - 1);
    float height = space * sqrt(3) / 2;
    for (uint i = 0; i < count; ++i) {
        set_thread(i, count);
        createTrianglesD(reinterpret_cast<float2*>(pos), id, loc, type, make_float2(px, py), N,
                         ntypes, typeVec, space, height, startID, count);
    }
}

}  /* extern "C" */
