// C ABI of the DEM step (include/demso_b200.h): argument checking, the
// per-stage entry points, and the context that runs the fused, graph-captured
// step on library-owned buffers.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "dem_common.cuh"
#include "dem_incsort.cuh"
#include "dem_kernels.cuh"
#include "dem_resident.cuh"
#include "dem_sort.cuh"

using namespace dem;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? DEM_ERR_NO_MEMORY : DEM_ERR_CUDA, "%s: %s", what,
                cudaGetErrorString(e));
}

// Every device allocation of the contexts goes through dev_alloc/dev_free,
// which count the allocations held and can be told to fail one
// (dem_debug_fail_allocation), so that tests can check that a failed create
// releases everything it took.
std::atomic<long long> g_liveAllocs{0};
std::atomic<int> g_failCountdown{0};

template <typename T>
cudaError_t dev_alloc(T** p, size_t bytes) {
    *p = nullptr;
    int k = g_failCountdown.load();
    while (k > 0 && !g_failCountdown.compare_exchange_weak(k, k - 1)) {
    }
    if (k == 1) return cudaErrorMemoryAllocation;  // the injected failure
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, bytes);
    if (e == cudaSuccess) {
        *p = static_cast<T*>(q);
        ++g_liveAllocs;
    }
    return e;
}

void dev_free(void* p) {
    if (!p) return;
    cudaFree(p);
    --g_liveAllocs;
}

#define DEM_TRY_CUDA(expr, what)                          \
    do {                                                  \
        cudaError_t _e = (expr);                          \
        if (_e != cudaSuccess) return cuda_fail(_e, what); \
    } while (0)

inline bool is_pow2(uint32_t v) { return v != 0 && (v & (v - 1u)) == 0; }

uint32_t log2_u32(uint32_t v) {
    uint32_t b = 0;
    while ((1ull << b) < (uint64_t)v) ++b;
    return b;
}

int validate(const DemSystem* s) {
    if (!s) return fail(DEM_ERR_INVALID_ARG, "system is NULL");
    if (!is_pow2(s->gridSize[0]) || !is_pow2(s->gridSize[1]))
        return fail(DEM_ERR_INVALID_ARG, "gridSize (%u, %u) must be powers of two",
                    s->gridSize[0], s->gridSize[1]);
    if ((uint64_t)s->gridSize[0] * s->gridSize[1] > (1ull << 31))
        return fail(DEM_ERR_INVALID_ARG, "too many cells");
    if (!(s->cubeDimension[0] > 0.0f) || !(s->cubeDimension[1] > 0.0f))
        return fail(DEM_ERR_INVALID_ARG, "cubeDimension must be positive");
    if (s->numMaterials < 1 || s->numMaterials > DEM_MAX_MATERIALS)
        return fail(DEM_ERR_INVALID_ARG, "numMaterials %u outside 1..%d", s->numMaterials,
                    DEM_MAX_MATERIALS);
    return DEM_OK;
}

// Host-side evaluation of the per-pair coefficients, with the reference's
// float expressions (particles_kernel.cuh:269-275, :417-421).
KParams make_kparams(const DemSystem* s, uint32_t n) {
    KParams P;
    memset(&P, 0, sizeof(P));
    P.n = n;
    P.gx = s->gridSize[0];
    P.gy = s->gridSize[1];
    P.gxf = (float)s->gridSize[0];
    P.gyf = (float)s->gridSize[1];
    P.Lx = s->cubeDimension[0];
    P.Ly = s->cubeDimension[1];
    P.dt = s->timeStep;
    P.gravx = s->gravity[0];
    P.gravy = s->gravity[1];
    P.ktWall = s->boundaryShearStiffness;
    P.nmat = s->numMaterials;
    P.rmax = INFINITY;
    P.cellW = P.Lx / P.gxf;
    P.cellH = P.Ly / P.gyf;
    P.cullMargin = 4e-6f * (P.Lx > P.Ly ? P.Lx : P.Ly);
    P.invLx = 1.0f / P.Lx;
    P.invLy = 1.0f / P.Ly;
    P.cellOff = 0;
    P.log2gx = 0;
    while ((1u << P.log2gx) < P.gx) ++P.log2gx;
    P.cull = 0;
    for (uint32_t a = 0; a < P.nmat; ++a) {
        const DemMaterial& A = s->materials[a];
        P.cn[a] = A.normalDamping;
        P.eb[a] = A.boundaryDamping;
        P.mu[a] = A.frictionCoefficient;
        P.at[a] = A.attractCoefficient;
        P.ktw[a] = series_assoc(A.shearStiffness, s->boundaryShearStiffness);
        for (uint32_t b = 0; b < P.nmat; ++b) {
            const DemMaterial& B = s->materials[b];
            P.pair[a * P.nmat + b] = make_float4(
                series_assoc(A.normalStiffness, B.normalStiffness),
                series_assoc(A.shearStiffness, B.shearStiffness),
                series_assoc(A.normalDamping, B.normalDamping),
                (A.frictionCoefficient + B.frictionCoefficient) / 2.0f);
        }
    }
    return P;
}

// Culling bound: the largest radius, and whether culling is valid for this
// grid (at least 3 cells per axis, cells wider than any contact distance).
void set_rmax(KParams& P, float rmax) {
    P.rmax = rmax;
    P.cull = (std::isfinite(rmax) && P.gx >= 3 && P.gy >= 3 && P.cellW > 2.002f * rmax &&
              P.cellH > 2.002f * rmax)
                 ? 1u
                 : 0u;
}

template <typename T>
bool misaligned(const T* p, size_t a) { return ((uintptr_t)p % a) != 0; }

}  // namespace

// Error recording for entry points defined in other translation units.
int dem_record_error(int code, const char* msg) { return fail(code, "%s", msg); }

// ---------------------------------------------------------------------------
// library
// ---------------------------------------------------------------------------
extern "C" int dem_abi_version(void) { return DEM_ABI_VERSION; }

extern "C" const char* dem_last_error_string(void) { return g_last_error.c_str(); }

extern "C" int dem_validate_system(const DemSystem* sys) { return validate(sys); }

// ---------------------------------------------------------------------------
// per-stage entry points
// ---------------------------------------------------------------------------
extern "C" int dem_calc_hash(const DemSystem* sys, const float* pos, uint32_t* gridParticleIndex,
                             uint32_t* gridParticleHash, uint32_t numParticles, void* stream) {
    int rc = validate(sys);
    if (rc) return rc;
    if (numParticles && (!pos || !gridParticleHash || !gridParticleIndex))
        return fail(DEM_ERR_INVALID_ARG, "dem_calc_hash: NULL buffer");
    if (misaligned(pos, 8)) return fail(DEM_ERR_INVALID_ARG, "pos must be 8-byte aligned");
    const KParams P = make_kparams(sys, numParticles);
    DEM_TRY_CUDA(launch_calc_hash(P, reinterpret_cast<const float2*>(pos), gridParticleHash,
                                  gridParticleIndex, numParticles, (cudaStream_t)stream),
                 "calc_hash launch");
    return DEM_OK;
}

extern "C" size_t dem_sort_scratch_bytes(uint32_t numParticles, uint32_t keyBits) {
    return sort_scratch_bytes(numParticles, keyBits);
}

extern "C" int dem_sort_particles(uint32_t* hash, uint32_t* index, uint32_t n, uint32_t keyBits,
                                  void* scratch, size_t scratchBytes, void* stream) {
    if (keyBits > 32) return fail(DEM_ERR_INVALID_ARG, "keyBits %u > 32", keyBits);
    if (n == 0) return DEM_OK;
    if (!hash || !index) return fail(DEM_ERR_INVALID_ARG, "dem_sort_particles: NULL buffer");
    const size_t need = sort_scratch_bytes(n, keyBits);
    if (!scratch || scratchBytes < need)
        return fail(DEM_ERR_INVALID_ARG, "dem_sort_particles: scratch %zu bytes < %zu needed",
                    scratchBytes, need);
    if (misaligned((const char*)scratch, 256))
        return fail(DEM_ERR_INVALID_ARG, "scratch must be 256-byte aligned");
    const SortScratch s = carve_sort_scratch(scratch, n, keyBits);
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t *ko, *vo;
    DEM_TRY_CUDA(radix_sort_pairs(hash, index, n, keyBits, false, s, st, &ko, &vo, nullptr),
                 "radix sort");
    if (ko != hash) {
        DEM_TRY_CUDA(cudaMemcpyAsync(hash, ko, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st),
                     "sort copy-back");
        DEM_TRY_CUDA(cudaMemcpyAsync(index, vo, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st),
                     "sort copy-back");
    }
    return DEM_OK;
}

extern "C" int dem_reorder_data_and_find_cell_start(
    const DemSystem* sys, uint32_t* cellStart, uint32_t* cellEnd, float* sortedPos,
    float* sortedVel, float* sortedTheta, float* sortedOmega, float* sortedRadius,
    float* sortedMass, uint32_t* sortedID, uint32_t* sortedLoc, uint32_t* sortedType,
    const uint32_t* hash, const uint32_t* index, const float* oldPos, const float* oldVel,
    const float* oldTheta, const float* oldOmega, const float* oldRadius, const float* oldMass,
    const uint32_t* oldID, const uint32_t* oldType, uint32_t numParticles, uint32_t numCells,
    void* stream) {
    int rc = validate(sys);
    if (rc) return rc;
    if (numCells != sys->gridSize[0] * sys->gridSize[1])
        return fail(DEM_ERR_INVALID_ARG, "numCells %u != gridSize product", numCells);
    if (!cellStart || !cellEnd) return fail(DEM_ERR_INVALID_ARG, "NULL cell arrays");
    if (numParticles &&
        (!sortedPos || !sortedVel || !sortedTheta || !sortedOmega || !sortedRadius ||
         !sortedMass || !sortedID || !sortedLoc || !hash || !index || !oldPos || !oldVel ||
         !oldTheta || !oldOmega || !oldRadius || !oldMass || !oldID))
        return fail(DEM_ERR_INVALID_ARG, "dem_reorder: NULL buffer");
    if ((sortedType == nullptr) != (oldType == nullptr))
        return fail(DEM_ERR_INVALID_ARG, "sortedType and oldType must both be set or both NULL");
    if (misaligned(sortedPos, 8) || misaligned(sortedVel, 8) || misaligned(oldPos, 8) ||
        misaligned(oldVel, 8))
        return fail(DEM_ERR_INVALID_ARG, "float2 arrays must be 8-byte aligned");
    const KParams P = make_kparams(sys, numParticles);
    DynSet s{reinterpret_cast<float2*>(sortedPos), reinterpret_cast<float2*>(sortedVel),
             sortedTheta, sortedOmega};
    StatSet sS{sortedRadius, sortedMass, sortedID, sortedType};
    DynSet o{const_cast<float2*>(reinterpret_cast<const float2*>(oldPos)),
             const_cast<float2*>(reinterpret_cast<const float2*>(oldVel)),
             const_cast<float*>(oldTheta), const_cast<float*>(oldOmega)};
    StatSet oS{const_cast<float*>(oldRadius), const_cast<float*>(oldMass),
               const_cast<uint32_t*>(oldID), const_cast<uint32_t*>(oldType)};
    DEM_TRY_CUDA(launch_reorder(P, cellStart, cellEnd, s, sS, sortedLoc, hash, index, o, oS,
                                numParticles, numCells, true, (cudaStream_t)stream, nullptr),
                 "reorder launch");
    return DEM_OK;
}

extern "C" int dem_collide(const DemSystem* sys, const float* pos, const float* vel, float* acc,
                           const float* omega, float* alpha, const uint32_t* type,
                           const float* radius, const float* mass, const uint32_t* cellStart,
                           const uint32_t* cellEnd, uint32_t numParticles, uint32_t numCells,
                           float* pressure, void* stream) {
    int rc = validate(sys);
    if (rc) return rc;
    if (numCells != sys->gridSize[0] * sys->gridSize[1])
        return fail(DEM_ERR_INVALID_ARG, "numCells %u != gridSize product", numCells);
    if (numParticles &&
        (!pos || !vel || !acc || !omega || !alpha || !radius || !mass || !cellStart || !cellEnd))
        return fail(DEM_ERR_INVALID_ARG, "dem_collide: NULL buffer");
    if (sys->numMaterials > 1 && !type)
        return fail(DEM_ERR_INVALID_ARG, "type array required with more than one material");
    if (misaligned(pos, 8) || misaligned(vel, 8) || misaligned(acc, 8))
        return fail(DEM_ERR_INVALID_ARG, "float2 arrays must be 8-byte aligned");
    const KParams P = make_kparams(sys, numParticles);
    DEM_TRY_CUDA(launch_collide(P, reinterpret_cast<const float2*>(pos),
                                reinterpret_cast<const float2*>(vel), omega, radius, mass, type,
                                cellStart, cellEnd, reinterpret_cast<float2*>(acc), alpha,
                                pressure, numParticles, (cudaStream_t)stream),
                 "collide launch");
    return DEM_OK;
}

extern "C" int dem_integrate_system(const DemSystem* sys, float* pos, float* vel,
                                    const float* acc, float* theta, float* omega,
                                    const float* alpha, const uint32_t* type, const float* radius,
                                    const float* mass, float* pressure, uint32_t numParticles,
                                    void* stream) {
    int rc = validate(sys);
    if (rc) return rc;
    if (numParticles && (!pos || !vel || !acc || !theta || !omega || !alpha || !radius || !mass))
        return fail(DEM_ERR_INVALID_ARG, "dem_integrate_system: NULL buffer");
    if (sys->numMaterials > 1 && !type)
        return fail(DEM_ERR_INVALID_ARG, "type array required with more than one material");
    if (misaligned(pos, 8) || misaligned(vel, 8) || misaligned(acc, 8))
        return fail(DEM_ERR_INVALID_ARG, "float2 arrays must be 8-byte aligned");
    const KParams P = make_kparams(sys, numParticles);
    DEM_TRY_CUDA(launch_integrate(P, reinterpret_cast<float2*>(pos), reinterpret_cast<float2*>(vel),
                                  reinterpret_cast<const float2*>(acc), theta, omega, alpha, type,
                                  radius, mass, pressure, numParticles, (cudaStream_t)stream),
                 "integrate launch");
    return DEM_OK;
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
struct DemContext {
    DemSystem sys;
    KParams P;
    uint32_t capacity = 0, n = 0, flags = 0, numCells = 0, keyBits = 0;
    // Row window (dem_create_rows): the context's cells are the scene's rows
    // rowFirst .. rowFirst + rows - 1; rows 0 for the whole grid.
    uint32_t rowFirst = 0, rows = 0;
    int device = 0;
    bool typed = false;
    // The current state (order of the last sort): positions in dyn[0].pos,
    // velocities, angles and spins in dyn[cur], the static fields in
    // stat[cur].  A step's sort moves positions into dyn[1].pos and radii
    // into stat[cur ^ 1] and records src; its step kernel gathers the other
    // fields through src and writes the new state into dyn[0].pos,
    // dyn[cur ^ 1] and stat[cur ^ 1].
    DynSet dyn[2];
    StatSet stat[2];
    int cur = 0;               // parity of the sets holding the current state
    uint32_t* src = nullptr;   // per sorted slot: the particle's slot in the previous order
    uint32_t* loc = nullptr;   // indexed by id
    uint32_t* keys = nullptr;  // cell of each particle of the current state
    uint32_t* perm = nullptr;  // radix sort values (full path)
    uint32_t* skey[2] = {};    // sorted keys of the order made when stat[p] was filled
    uint2* cells[2] = {};      // interleaved (cellStart, cellEnd) of that order
    uint32_t* first[2] = {};   // first particle of every cell of that order (numCells + 4)
    float* pressure = nullptr;
    float2* acc = nullptr;
    float* alpha = nullptr;
    uint32_t* errFlag = nullptr;
    void* sortScratch = nullptr;
    OnesweepScratch ss;
    void* incScratch = nullptr;
    IncSort inc;
    // batched form: specimen table (device + host copy), slot -> specimen,
    // first slot of every specimen (nspec + 1 entries)
    uint32_t nspec = 0;
    KParams* dTable = nullptr;
    std::vector<KParams> hTable;
    uint32_t* spec = nullptr;
    std::vector<uint32_t> partOff;
    // the control particle (dem_set_control): device state, reaction vectors
    // (3 n floats), block partials and the reaction of the last step
    bool ctlOn = false;
    void* ctlBlock = nullptr;
    ControlDev* dCtl = nullptr;
    float* ctlVec = nullptr;
    float* ctlPartials = nullptr;
    float* ctlOut = nullptr;
    // dem_render's per-pixel owner scratch
    uint32_t* renderOwner = nullptr;
    size_t renderOwnerWords = 0;
    bool keysValid = false;  // keys[] holds the cell of every particle of the current state
    bool haveOrder = false;  // the last step recorded its movers: incremental sort possible
    bool inSortOrder = false;  // the state is in the order of its last sort (skey/first[cur])
    float rmax = INFINITY;   // largest radius of the current state (culling bound)
    cudaStream_t capStream = nullptr, bodyStream = nullptr;
    // capture-time fork of the sort phase: the full path's branch
    cudaStream_t forkStream = nullptr;
    cudaEvent_t forkEv = nullptr, joinEv = nullptr;
    // the incremental sort's movers, placed beside its stayers
    cudaStream_t moverStream = nullptr;
    cudaEvent_t moverForkEv = nullptr, moverJoinEv = nullptr;
    // The device-side step loop of multi-step dem_step calls: loopGraph[p]
    // runs pairs of incremental steps from parity p in a WHILE node while the
    // count in loopCtl[1] (copied from loopCtl[0], written before each launch)
    // is non-zero; its body is captured on loopStream.
    cudaGraphExec_t loopGraph[2] = {};
    uint32_t* loopCtl = nullptr;
    cudaStream_t loopStream = nullptr;
    // Each step is two graph launches: the sort phase sortGraph[kind][parity]
    // (kind 0 = full radix sort, 1 = incremental sort with the full sort as a
    // device-chosen fallback), then the step kernel stepGraph[parity].
    cudaGraphExec_t sortGraph[2][2] = {};
    cudaGraphExec_t stepGraph[2] = {};
    int launchesPerStep = 0;
    void* block = nullptr;  // one allocation for every per-particle/per-cell array
    // followed-particle staging (device), see dem_get_followed
    float* followRows = nullptr;
    // dem_step_followed: the ids (device copy), the ring of per-step rows,
    // and its device-side loop followGraph[parity] (holds both pointers)
    uint32_t* followIds = nullptr;
    uint32_t followIdsCap = 0;
    float* followRing = nullptr;
    size_t followRingBytes = 0;
    std::vector<uint32_t> followIdsHost;
    cudaGraphExec_t followGraph[2] = {};
    // stage profiling: events recorded on the caller's stream around the two
    // launches of each step (3 per step)
    bool profiling = false;
    cudaEvent_t* evPool = nullptr;
    uint32_t evCap = 0, evUsed = 0, stepsProfiled = 0;
    // adjoint: checkpoints of the state every adjEvery steps of the last
    // dem_adj_forward (pos, vel, theta, omega, radius, mass, id per slot)
    void* adjCheck = nullptr;
    size_t adjCheckBytes = 0;
    uint32_t adjSteps = 0, adjEvery = 0, adjWindows = 0;
    uint32_t adjN = 0;     // particles and largest radius of the checkpointed run
    float adjRmax = 0.0f;  // (the backward restores checkpoints without re-deriving them)
    // dem_adj_backward's buffers (the window's per-step record, the tangent
    // and reduction scratch), kept across calls and grown on demand, and its
    // two loops (recompute pairs of each parity, reverse steps), kept while
    // the buffers, the record's layout and the caller's cotangent buffers
    // they were captured with are unchanged
    // DEM_CTX_RESIDENT (batches): the specimens packed into bins, the bins'
    // queue word and the blocks' scratch, made at the first resident call;
    // resPlanned with resBins == 0 means the batch does not fit (a specimen
    // too large for one bin), and the graph path steps it
    bool resPlanned = false;
    uint32_t resBins = 0, resMaxN = 0, resMaxC = 0;
    int resBlocks = 0;
    ResBin* dResBins = nullptr;
    ResEntry* dResEntries = nullptr;
    uint32_t* resQueue = nullptr;
    void* resWork = nullptr;
    // DEM_CTX_RESIDENT (single scenes): the cluster launch's scratch, and
    // whether a cluster of its shape could not be made resident here
    void* clusterWork = nullptr;
    size_t clusterWorkBytes = 0;
    bool clusterUnsupported = false;
    void* adjRec = nullptr;
    size_t adjRecBytes = 0;
    void* adjTmp = nullptr;
    size_t adjTmpBytes = 0;
    cudaGraphExec_t adjRecLoop[2] = {};
    cudaGraphExec_t adjRevLoop = nullptr;
    const void* adjRevKey[3] = {};
    size_t adjRevStepBytes = 0;
    uint32_t adjRevN = 0;
    // the step kernel's launch shape (step_variant_shape) and its autotuner
    // (DEM_CTX_AUTOTUNE): the first kTuneSteps steps run the variants in turn,
    // each timed by a pair of events, then the one with the smallest median
    // is kept.  tuned: 1 chosen by the tuner, 0 fixed, -1 still timing.
    int variant = 0;
    int tuned = 0;
    uint32_t tuneStep = 0;
    cudaGraphExec_t tuneGraph[kStepVariants][2] = {};
    cudaEvent_t* tuneEv = nullptr;
    float tuneMs[kStepVariants] = {};
};

namespace {

// Kernel parameters of a single-scene context over `n` particles: the
// scene's, with a row window's row count and first row.
KParams scene_kparams(const DemContext* c, uint32_t n) {
    KParams P = make_kparams(&c->sys, n);
    if (c->rows) {
        P.gy = c->rows;
        P.rowOff = (int32_t)c->rowFirst;
    }
    return P;
}

// rounds of the autotuner: every variant once per round, the first round
// (cold instruction caches, first graph launches) not counted
constexpr uint32_t kTuneRounds = 6;
constexpr uint32_t kTuneSteps = kTuneRounds * kStepVariants;

void drop_tune_graphs(DemContext* c) {
    for (int v = 0; v < kStepVariants; ++v)
        for (int p = 0; p < 2; ++p) {
            if (c->tuneGraph[v][p]) cudaGraphExecDestroy(c->tuneGraph[v][p]);
            c->tuneGraph[v][p] = nullptr;
        }
}

void drop_adj_graphs(DemContext* c) {
    for (int p = 0; p < 2; ++p) {
        if (c->adjRecLoop[p]) cudaGraphExecDestroy(c->adjRecLoop[p]);
        c->adjRecLoop[p] = nullptr;
    }
    if (c->adjRevLoop) cudaGraphExecDestroy(c->adjRevLoop);
    c->adjRevLoop = nullptr;
}

void drop_loop_graphs(DemContext* c) {
    for (int p = 0; p < 2; ++p) {
        if (c->loopGraph[p]) cudaGraphExecDestroy(c->loopGraph[p]);
        c->loopGraph[p] = nullptr;
        if (c->followGraph[p]) cudaGraphExecDestroy(c->followGraph[p]);
        c->followGraph[p] = nullptr;
    }
    drop_adj_graphs(c);
}

void drop_graphs(DemContext* c) {
    drop_tune_graphs(c);
    drop_loop_graphs(c);
    // a tuning interrupted by a change of the step starts again
    if (c->tuned < 0) c->tuneStep = 0;
    for (int k = 0; k < 2; ++k)
        for (int p = 0; p < 2; ++p) {
            if (c->sortGraph[k][p]) cudaGraphExecDestroy(c->sortGraph[k][p]);
            c->sortGraph[k][p] = nullptr;
        }
    for (int p = 0; p < 2; ++p) {
        if (c->stepGraph[p]) cudaGraphExecDestroy(c->stepGraph[p]);
        c->stepGraph[p] = nullptr;
    }
}

MoverSinkArgs sink_of(DemContext* c) {
    MoverSinkArgs m;
    m.leavers = c->inc.leavers;
    m.arrCnt = c->inc.arrCnt;
    m.arrLo = c->inc.arrLo;
    m.movers = c->inc.movers;
    m.ctrl = c->inc.ctrl;
    m.moverCap = c->inc.moverCap;
    m.tileShift = c->inc.tileShift;
    m.dirty = c->inc.dirty;
    return m;
}

// Full sort of the current state (parity a) into the other static set.
// What the sort phase of parity a moves: positions and radii into the
// sorted order, with the previous slot of every sorted slot.
SortMove sort_move(DemContext* c, int a) {
    return SortMove{c->dyn[0].pos, c->stat[a].radius, c->dyn[1].pos, c->stat[a ^ 1].radius,
                    c->src};
}

cudaError_t enqueue_full_sort(DemContext* c, int a, cudaStream_t st, int* launches) {
    const int b = a ^ 1;
    return enqueue_full(c->inc, c->n, c->keyBits, c->keys, c->perm, c->ss, c->errFlag, c->skey[b],
                        c->cells[b], c->first[b], sort_move(c, a), st, launches);
}

cudaError_t enqueue_inc_tail(DemContext* c, int a, cudaStream_t st, int* launches) {
    const int b = a ^ 1;
    return enqueue_incremental_tail(c->inc, c->n, c->keys, c->skey[a], c->cells[a], c->first[a],
                                    c->skey[b], c->cells[b], c->first[b], sort_move(c, a), st,
                                    launches, c->moverStream, c->moverForkEv, c->moverJoinEv);
}

// The incremental sort launched directly (the host chose it).
cudaError_t enqueue_inc_sort(DemContext* c, int a, cudaStream_t st, int* launches) {
    cudaError_t e = enqueue_incremental_head(c->inc, c->cells[a], c->first[a], 0, false, st,
                                             launches);
    return e == cudaSuccess ? enqueue_inc_tail(c, a, st, launches) : e;
}

// Adds a conditional node of `type` on `h` at the current capture point of
// `st` and captures `body` into it on `bodyStream`.
template <typename Body>
cudaError_t add_conditional(cudaStream_t st, cudaGraphConditionalHandle h,
                            cudaGraphConditionalNodeType type, cudaStream_t bodyStream,
                            Body body) {
    cudaStreamCaptureStatus status;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &status, nullptr, &g, &deps, &nd);
    if (e != cudaSuccess) return e;
    cudaGraphNodeParams prm = {};
    prm.type = cudaGraphNodeTypeConditional;
    prm.conditional.handle = h;
    prm.conditional.type = type;
    prm.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, g, deps, nd, &prm);
    if (e != cudaSuccess) return e;
    e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
    if (e != cudaSuccess) return e;
    cudaGraph_t bodyGraph = prm.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(bodyStream, bodyGraph, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    cudaError_t eb = body(bodyStream);
    e = cudaStreamEndCapture(bodyStream, &bodyGraph);
    return eb != cudaSuccess ? eb : e;
}

template <typename Body>
cudaError_t add_if(DemContext* c, cudaStream_t st, cudaGraphConditionalHandle h, Body body) {
    return add_conditional(st, h, cudaGraphCondTypeIf, c->bodyStream, body);
}

// Sort phase of one step: the state (dyn[0], stat[cur]) is sorted into
// (dyn[1], stat[cur^1]) with its cell ranges.  kind 0: full radix sort;
// kind 1: incremental sort, or the full sort when the last step's movers did
// not fit.  In kind 1 the incremental kernels are plain graph nodes that
// return at once when the full path is due, and the full path is the body of
// one conditional node on a branch beside them, forked after the first
// incremental kernel (which sets its condition): when the node does not run
// its body, evaluating it overlaps the incremental kernels instead of adding
// to the step.  The two branches never both do work in one step.
cudaError_t enqueue_sort_phase(DemContext* c, int kind, cudaStream_t st, int* launches) {
    const int a = c->cur;
    if (kind == 0) return enqueue_full_sort(c, a, st, launches);
    cudaStreamCaptureStatus status;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &status, nullptr, &g, nullptr, nullptr);
    if (e != cudaSuccess) return e;
    if (status != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureUnsupported;
    cudaGraphConditionalHandle hFull;
    e = cudaGraphConditionalHandleCreate(&hFull, g, 0, cudaGraphCondAssignDefault);
    if (e == cudaSuccess)
        e = enqueue_incremental_head(c->inc, c->cells[a], c->first[a], hFull, true, st, launches);
    if (e != cudaSuccess) return e;
    e = cudaEventRecord(c->forkEv, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->forkStream, c->forkEv, 0);
    if (e != cudaSuccess) return e;
    int fullLaunches = 0;
    e = add_if(c, c->forkStream, hFull, [&](cudaStream_t bs) {
        return enqueue_full_sort(c, a, bs, &fullLaunches);
    });
    cudaError_t ej = cudaEventRecord(c->joinEv, c->forkStream);
    if (e == cudaSuccess) e = ej;
    if (e == cudaSuccess) e = enqueue_inc_tail(c, a, st, launches);
    ej = cudaStreamWaitEvent(st, c->joinEv, 0);  // join the branch even after an error
    return e == cudaSuccess ? ej : e;
}

// Collide + integrate + next hash over the sorted set made by the sort phase.
// The inputs of the step kernel of parity a: sorted positions and radii, the
// other fields in the previous order (gathered through src).
DynSet step_in(DemContext* c, int a) {
    return DynSet{c->dyn[1].pos, c->dyn[a].vel, c->dyn[a].theta, c->dyn[a].omega};
}
StatSet step_in_static(DemContext* c, int a) {
    return StatSet{c->stat[a ^ 1].radius, c->stat[a].mass, c->stat[a].id, c->stat[a].type};
}
// The current state (order of the last sort), see DemContext.
DynSet state_dyn(DemContext* c) {
    return DynSet{c->dyn[0].pos, c->dyn[c->cur].vel, c->dyn[c->cur].theta, c->dyn[c->cur].omega};
}

cudaError_t enqueue_step_kernel(DemContext* c, cudaStream_t st, int* launches) {
    const int a = c->cur, b = a ^ 1;
    ControlArgs ctl{};
    if (c->ctlOn) ctl = ControlArgs{c->dCtl, c->ctlVec, c->ctlVec + c->capacity,
                                    c->ctlVec + 2ull * c->capacity};
    const DynSet out{c->dyn[0].pos, c->dyn[b].vel, c->dyn[b].theta, c->dyn[b].omega};
    cudaError_t e = launch_step(c->P, step_in(c, a), step_in_static(c, a), c->src, c->skey[b],
                                c->cells[b], c->first[b], out, c->stat[b], c->loc,
                                c->keys, (c->flags & DEM_CTX_PRESSURE) ? c->pressure : nullptr,
                                (c->flags & DEM_CTX_ACCEL) ? c->acc : nullptr,
                                (c->flags & DEM_CTX_ACCEL) ? c->alpha : nullptr, c->errFlag, c->n,
                                sink_of(c), st, c->nspec ? c->dTable : nullptr, c->spec, ctl,
                                c->variant);
    if (launches) ++*launches;
    if (e == cudaSuccess && c->ctlOn)
        e = launch_control_post(ctl, c->dCtl, c->n, c->ctlPartials, c->ctlOut, st, launches);
    return e;
}

// what: 0/1 = sort phase of that kind, 2 = step kernel (of c->variant's
// shape), 3 = the step kernel into the autotuner's graph of c->variant.
int build_graph(DemContext* c, int what, int parity) {
    cudaGraph_t g = nullptr;
    const int saved = c->cur;
    c->cur = parity;
    DEM_TRY_CUDA(cudaStreamBeginCapture(c->capStream, cudaStreamCaptureModeThreadLocal),
                 "begin capture");
    int launches = 0;
    cudaError_t e = what < 2 ? enqueue_sort_phase(c, what, c->capStream, &launches)
                             : enqueue_step_kernel(c, c->capStream, &launches);
    cudaError_t e2 = cudaStreamEndCapture(c->capStream, &g);
    c->cur = saved;
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return cuda_fail(e, "step capture");
    }
    if (e2 != cudaSuccess) return cuda_fail(e2, "end capture");
    cudaGraphExec_t* slot = what < 2    ? &c->sortGraph[what][parity]
                            : what == 2 ? &c->stepGraph[parity]
                                        : &c->tuneGraph[c->variant][parity];
    e = cudaGraphInstantiate(slot, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "graph instantiate");
    if (what == 1) c->launchesPerStep = launches + 1 + (c->ctlOn ? 2 : 0);  // + the step graph
    return DEM_OK;
}

// Device-side loop control words (loopCtl, written by the host before each
// launch of a loop graph): the requested count, the count left, the slot.
enum : uint32_t {
    kLoopStepReq = 0, kLoopStepLeft = 1,                    // dem_step's step pairs
    kLoopRecReq = 2, kLoopRecLeft = 3, kLoopRecSlot = 4,    // adjoint recompute pairs
    kLoopRevReq = 5, kLoopRevLeft = 6, kLoopRevSlot = 7,    // adjoint reversed steps
    kLoopFolReq = 8, kLoopFolLeft = 9, kLoopFolSlot = 10,   // dem_step_followed pairs
    kLoopFolCount = 11,                                     // its number of ids
};

// A graph of one device-side loop: an init kernel that copies loopCtl[req]
// to loopCtl[req + 1] and sets the condition, then a WHILE node whose body
// is `body` (captured on loopStream) followed by the kernel that counts one
// iteration down and adds idxStep to loopCtl[idx] (idx < 0: none).
template <typename Body>
int build_while_graph(DemContext* c, uint32_t req, int idx, int32_t idxStep, Body body,
                      cudaGraphExec_t* out) {
    const int saved = c->cur;
    DEM_TRY_CUDA(cudaStreamBeginCapture(c->capStream, cudaStreamCaptureModeThreadLocal),
                 "begin capture");
    cudaStreamCaptureStatus status;
    cudaGraph_t cg = nullptr;
    cudaGraphConditionalHandle h = 0;
    uint32_t* left = c->loopCtl + req + 1;
    uint32_t* slot = idx < 0 ? nullptr : c->loopCtl + idx;
    cudaError_t e = cudaStreamGetCaptureInfo(c->capStream, &status, nullptr, &cg, nullptr, nullptr);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, cg, 0, 0);
    if (e == cudaSuccess) e = launch_loop_init(c->loopCtl + req, left, h, c->capStream);
    if (e == cudaSuccess)
        e = add_conditional(c->capStream, h, cudaGraphCondTypeWhile, c->loopStream,
                            [&](cudaStream_t bs) {
                                cudaError_t eb = body(bs);
                                if (eb == cudaSuccess) eb = launch_loop_next(left, slot, idxStep, h, bs);
                                return eb;
                            });
    c->cur = saved;
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(c->capStream, &g);
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return cuda_fail(e, "loop capture");
    }
    if (e2 != cudaSuccess) return cuda_fail(e2, "end capture");
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "loop instantiate");
    return DEM_OK;
}

// Two incremental steps from parity p (p, then p ^ 1: the sort phase and the
// step kernel as in sortGraph[1] and stepGraph) into `bs`, each followed by
// after(k, bs) (k = 0, 1: the step's place in the pair).
template <typename After>
cudaError_t enqueue_step_pair(DemContext* c, int p, cudaStream_t bs, After after) {
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        c->cur = p ^ k;
        e = enqueue_sort_phase(c, 1, bs, nullptr);
        if (e == cudaSuccess) e = enqueue_step_kernel(c, bs, nullptr);
        if (e == cudaSuccess) e = after(k, bs);
    }
    return e;
}

// dem_step's loop from parity p: pairs of steps while loopCtl[kLoopStepLeft].
int build_loop_graph(DemContext* c, int p) {
    return build_while_graph(
        c, kLoopStepReq, -1, 0,
        [&](cudaStream_t bs) {
            return enqueue_step_pair(c, p, bs, [](int, cudaStream_t) { return cudaSuccess; });
        },
        &c->loopGraph[p]);
}

// The followed rows of the state after a step of parity a (the current
// state is then dyn[0].pos, dyn[a ^ 1], stat[a ^ 1]) into ring block
// (slot ? *slot : 0) + add.
cudaError_t enqueue_followed_ring(DemContext* c, int a, const uint32_t* slot, uint32_t add,
                                  cudaStream_t st) {
    const int b = a ^ 1;
    return launch_followed_ring(c->followIds, c->loopCtl + kLoopFolCount, slot, add, c->loc,
                                DynSet{c->dyn[0].pos, c->dyn[b].vel, c->dyn[b].theta, c->dyn[b].omega},
                                c->stat[b], (c->flags & DEM_CTX_ACCEL) ? c->acc : nullptr,
                                (c->flags & DEM_CTX_ACCEL) ? c->alpha : nullptr,
                                (c->flags & DEM_CTX_PRESSURE) ? c->pressure : nullptr,
                                c->followRing, st);
}

// dem_step_followed's loop from parity p: pairs of steps, each followed by
// its rows at ring block loopCtl[kLoopFolSlot] + k.
int build_follow_graph(DemContext* c, int p) {
    return build_while_graph(
        c, kLoopFolReq, kLoopFolSlot, 2,
        [&](cudaStream_t bs) {
            return enqueue_step_pair(c, p, bs, [&](int k, cudaStream_t s2) {
                return enqueue_followed_ring(c, p ^ k, c->loopCtl + kLoopFolSlot, (uint32_t)k, s2);
            });
        },
        &c->followGraph[p]);
}

void drop_tune_events(DemContext* c) {
    if (!c->tuneEv) return;
    for (uint32_t i = 0; i < 2 * kTuneSteps; ++i)
        if (c->tuneEv[i]) cudaEventDestroy(c->tuneEv[i]);
    delete[] c->tuneEv;
    c->tuneEv = nullptr;
}

// Before a tuning step: the events (and, on the graph path, every variant's
// step graph) exist.
int tune_prepare(DemContext* c, bool graphs) {
    if (!c->tuneEv) {
        c->tuneEv = new (std::nothrow) cudaEvent_t[2 * kTuneSteps]();
        if (!c->tuneEv) return fail(DEM_ERR_NO_MEMORY, "host allocation failed");
        for (uint32_t i = 0; i < 2 * kTuneSteps; ++i)
            DEM_TRY_CUDA(cudaEventCreate(&c->tuneEv[i]), "tuner event");
    }
    if (!graphs) return DEM_OK;
    const int keep = c->variant;
    for (int v = 0; v < kStepVariants; ++v)
        for (int p = 0; p < 2; ++p)
            if (!c->tuneGraph[v][p]) {
                c->variant = v;
                const int rc = build_graph(c, 3, p);
                c->variant = keep;
                if (rc) return rc;
            }
    return DEM_OK;
}

// After the last tuning step: the median time of each variant, the fastest
// kept (the lower index on a tie), its graphs moved into stepGraph.
int tune_finish(DemContext* c, bool graphs) {
    DEM_TRY_CUDA(cudaEventSynchronize(c->tuneEv[2 * kTuneSteps - 1]), "tuner sync");
    int best = 0;
    for (int v = 0; v < kStepVariants; ++v) {
        float t[kTuneRounds - 1];
        for (uint32_t r = 1; r < kTuneRounds; ++r) {
            const uint32_t s = r * kStepVariants + (uint32_t)v;
            DEM_TRY_CUDA(cudaEventElapsedTime(&t[r - 1], c->tuneEv[2 * s], c->tuneEv[2 * s + 1]),
                         "tuner time");
        }
        std::sort(t, t + (kTuneRounds - 1));
        c->tuneMs[v] = t[(kTuneRounds - 1) / 2];
        if (c->tuneMs[v] < c->tuneMs[best]) best = v;
    }
    c->variant = best;
    c->tuned = 1;
    if (graphs)
        for (int p = 0; p < 2; ++p) {
            if (c->stepGraph[p]) cudaGraphExecDestroy(c->stepGraph[p]);
            c->stepGraph[p] = c->tuneGraph[best][p];
            c->tuneGraph[best][p] = nullptr;
        }
    drop_tune_graphs(c);
    drop_tune_events(c);
    drop_loop_graphs(c);  // they hold the step kernel of the old shape
    return DEM_OK;
}

void drop_profile(DemContext* c) {
    if (c->evPool) {
        for (uint32_t i = 0; i < c->evCap; ++i) cudaEventDestroy(c->evPool[i]);
        delete[] c->evPool;
        c->evPool = nullptr;
    }
    c->evCap = c->evUsed = 0;
    c->profiling = false;
}

size_t al256(size_t b) { return (b + 255u) & ~(size_t)255u; }

}  // namespace

// Allocates the buffers of a context of `capacity` particles over `numCells`
// cells (c->sys, c->P, c->typed and c->flags already set).
int init_context(DemContext* c, uint32_t capacity, uint32_t numCells, DemContext** out);

extern "C" int dem_create(const DemSystem* sys, uint32_t capacity, uint32_t flags,
                          DemContext** out) {
    if (!out) return fail(DEM_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    int rc = validate(sys);
    if (rc) return rc;
    return dem_create_rows(sys, capacity, flags, 0, sys->gridSize[1], out);
}

extern "C" int dem_create_rows(const DemSystem* sys, uint32_t capacity, uint32_t flags,
                               uint32_t rowFirst, uint32_t rowCount, DemContext** out) {
    if (!out) return fail(DEM_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    int rc = validate(sys);
    if (rc) return rc;
    if (capacity == 0) return fail(DEM_ERR_INVALID_ARG, "capacity must be > 0");
    if (capacity >= (1u << 30)) return fail(DEM_ERR_INVALID_ARG, "capacity must be < 2^30");
    const uint32_t gy = sys->gridSize[1];
    if (!is_pow2(rowCount) || rowCount > gy)
        return fail(DEM_ERR_INVALID_ARG, "rowCount %u: a power of two, at most the grid's %u rows",
                    rowCount, gy);
    if (rowFirst >= gy)
        return fail(DEM_ERR_INVALID_ARG, "rowFirst %u outside the grid's %u rows", rowFirst, gy);
    DemContext* c = new (std::nothrow) DemContext();
    if (!c) return fail(DEM_ERR_NO_MEMORY, "host allocation failed");
    c->sys = *sys;
    c->flags = flags;
    c->typed = sys->numMaterials > 1;
    // the whole grid is no window: rows 0 keeps every kernel parameter the
    // scene's own
    if (rowFirst != 0 || rowCount != gy) {
        c->rowFirst = rowFirst;
        c->rows = rowCount;
    }
    c->P = scene_kparams(c, 0);
    return init_context(c, capacity, sys->gridSize[0] * rowCount, out);
}

extern "C" int dem_batch_create(const DemSystem* specs, uint32_t numSpecimens, uint32_t flags,
                                DemContext** out) {
    if (!out) return fail(DEM_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (!specs || numSpecimens == 0) return fail(DEM_ERR_INVALID_ARG, "no specimens");
    uint64_t total = 0, cells = 0;
    uint32_t nmat = 1;
    bool attract = false;
    for (uint32_t s = 0; s < numSpecimens; ++s) {
        int rc = validate(&specs[s]);
        if (rc) return rc;
        total += specs[s].numParticles;
        cells += (uint64_t)specs[s].gridSize[0] * specs[s].gridSize[1];
        nmat = std::max(nmat, specs[s].numMaterials);
        for (uint32_t m = 0; m < specs[s].numMaterials; ++m)
            attract = attract || specs[s].materials[m].attractCoefficient != 0.0f;
    }
    if (total == 0 || total >= (1u << 30)) return fail(DEM_ERR_INVALID_ARG, "batch size %llu", (unsigned long long)total);
    if (cells > (1ull << 31)) return fail(DEM_ERR_INVALID_ARG, "too many cells in the batch");
    DemContext* c = new (std::nothrow) DemContext();
    if (!c) return fail(DEM_ERR_NO_MEMORY, "host allocation failed");
    c->sys = specs[0];
    c->flags = flags;
    c->typed = nmat > 1;
    c->nspec = numSpecimens;
    c->hTable.resize(numSpecimens);
    c->partOff.assign(numSpecimens + 1, 0u);
    uint32_t cellOff = 0;
    for (uint32_t s = 0; s < numSpecimens; ++s) {
        c->hTable[s] = make_kparams(&specs[s], specs[s].numParticles);
        c->hTable[s].cellOff = cellOff;
        cellOff += specs[s].gridSize[0] * specs[s].gridSize[1];
        c->partOff[s + 1] = c->partOff[s] + specs[s].numParticles;
    }
    // the context-wide parameters only steer template choices: a material
    // count and an attraction flag that cover every specimen
    c->P = make_kparams(&specs[0], (uint32_t)total);
    c->P.nmat = nmat;
    c->P.at[0] = attract ? 1.0f : 0.0f;
    for (uint32_t m = 1; m < kMaxMat; ++m) c->P.at[m] = 0.0f;
    int rc = init_context(c, (uint32_t)total, (uint32_t)cells, out);
    if (rc) return rc;
    c = *out;
    std::vector<uint32_t> slotSpec(total);
    for (uint32_t s = 0; s < numSpecimens; ++s)
        for (uint32_t k = c->partOff[s]; k < c->partOff[s + 1]; ++k) slotSpec[k] = s;
    cudaError_t e = dev_alloc(&c->dTable, sizeof(KParams) * numSpecimens);
    if (e == cudaSuccess) e = dev_alloc(&c->spec, sizeof(uint32_t) * total);
    if (e == cudaSuccess)
        e = cudaMemcpy(c->dTable, c->hTable.data(), sizeof(KParams) * numSpecimens,
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(c->spec, slotSpec.data(), sizeof(uint32_t) * total, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        dem_destroy(c);
        *out = nullptr;
        return cuda_fail(e, "batch tables");
    }
    return DEM_OK;
}

extern "C" int dem_batch_specimen(DemContext* c, uint32_t specimen, uint32_t* firstSlot,
                                  uint32_t* count) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    if (!c->nspec) return fail(DEM_ERR_INVALID_ARG, "not a batch");
    if (specimen >= c->nspec) return fail(DEM_ERR_INVALID_ARG, "specimen %u >= %u", specimen, c->nspec);
    if (firstSlot) *firstSlot = c->partOff[specimen];
    if (count) *count = c->partOff[specimen + 1] - c->partOff[specimen];
    return DEM_OK;
}

int init_context(DemContext* c, uint32_t capacity, uint32_t numCells, DemContext** out) {
    c->tuned = (c->flags & DEM_CTX_AUTOTUNE) ? -1 : 0;
    c->capacity = capacity;
    c->numCells = numCells;
    c->keyBits = log2_u32(c->numCells);
    cudaGetDevice(&c->device);

    const size_t N = capacity, f4 = al256(4 * N), f8 = al256(8 * N),
                 cells8 = al256(8 * (size_t)c->numCells),
                 first4 = al256(4 * ((size_t)c->numCells + 4));
    // the sorted positions and radii are read up to kFilterPad - 1 elements
    // past the last particle by the step kernel's candidate filter
    const size_t f4p = al256(4 * (N + kFilterPad)), f8p = al256(8 * (N + kFilterPad));
    // the particle state: two dynamic and two static sets, unless the
    // caller's buffers are adopted instead (DEM_CTX_CALLER_STATE)
    const bool ownState = !(c->flags & DEM_CTX_CALLER_STATE);
    size_t total = 0;
    if (ownState) {
        total += 2 * (f8p + f8 + 2 * f4);                    // dyn sets
        total += 2 * (f4p + 2 * f4 + (c->typed ? f4 : 0));   // static sets
    }
    total += 4 * f4 + 2 * f4;                    // loc, keys, perm, src, sorted keys x2
    total += 2 * cells8 + 2 * first4;            // cell ranges and first particles x2
    total += f4 + f8 + f4;                       // pressure, acc, alpha
    total += 256;                                // error flag
    total += 256;                                // step-loop counters
    const size_t sortBytes = onesweep_scratch_bytes(capacity, c->keyBits);
    const size_t incBytes = incsort_bytes(capacity, c->numCells, nullptr);
    cudaError_t e = dev_alloc(&c->block, total);
    if (e == cudaSuccess) e = dev_alloc(&c->sortScratch, sortBytes);
    if (e == cudaSuccess) e = dev_alloc(&c->incScratch, incBytes);
    if (e != cudaSuccess) {
        dev_free(c->incScratch);
        dev_free(c->sortScratch);
        dev_free(c->block);
        delete c;
        return cuda_fail(e, "cudaMalloc context");
    }
    char* p = static_cast<char*>(c->block);
    auto take = [&p](size_t b) { char* q = p; p += b; return q; };
    for (int s = 0; s < 2 && ownState; ++s) {
        c->dyn[s].pos = reinterpret_cast<float2*>(take(f8p));
        c->dyn[s].vel = reinterpret_cast<float2*>(take(f8));
        c->dyn[s].theta = reinterpret_cast<float*>(take(f4));
        c->dyn[s].omega = reinterpret_cast<float*>(take(f4));
        c->stat[s].radius = reinterpret_cast<float*>(take(f4p));
        c->stat[s].mass = reinterpret_cast<float*>(take(f4));
        c->stat[s].id = reinterpret_cast<uint32_t*>(take(f4));
        c->stat[s].type = c->typed ? reinterpret_cast<uint32_t*>(take(f4)) : nullptr;
    }
    c->loc = reinterpret_cast<uint32_t*>(take(f4));
    c->keys = reinterpret_cast<uint32_t*>(take(f4));
    c->perm = reinterpret_cast<uint32_t*>(take(f4));
    c->src = reinterpret_cast<uint32_t*>(take(f4));
    for (int s = 0; s < 2; ++s) {
        c->skey[s] = reinterpret_cast<uint32_t*>(take(f4));
        c->cells[s] = reinterpret_cast<uint2*>(take(cells8));
        c->first[s] = reinterpret_cast<uint32_t*>(take(first4));
    }
    c->pressure = reinterpret_cast<float*>(take(f4));
    c->acc = reinterpret_cast<float2*>(take(f8));
    c->alpha = reinterpret_cast<float*>(take(f4));
    c->errFlag = reinterpret_cast<uint32_t*>(take(256));
    c->loopCtl = reinterpret_cast<uint32_t*>(take(256));
    c->ss = carve_onesweep_scratch(c->sortScratch, capacity, c->keyBits);
    c->inc = carve_incsort(c->incScratch, capacity, c->numCells);
    c->inc.errFlag = c->errFlag;
    e = cudaMemset(c->block, 0, total);
    if (e == cudaSuccess) e = cudaMemset(c->incScratch, 0, incBytes);
    for (int s = 0; s < 2 && e == cudaSuccess; ++s)
        e = cudaMemset(c->cells[s], 0xff, 8 * (size_t)c->numCells);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->capStream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->bodyStream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->forkStream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->loopStream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->forkEv, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->joinEv, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->moverStream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->moverForkEv, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->moverJoinEv, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        if (c->moverJoinEv) cudaEventDestroy(c->moverJoinEv);
        if (c->moverForkEv) cudaEventDestroy(c->moverForkEv);
        if (c->moverStream) cudaStreamDestroy(c->moverStream);
        if (c->joinEv) cudaEventDestroy(c->joinEv);
        if (c->forkEv) cudaEventDestroy(c->forkEv);
        if (c->loopStream) cudaStreamDestroy(c->loopStream);
        if (c->forkStream) cudaStreamDestroy(c->forkStream);
        if (c->bodyStream) cudaStreamDestroy(c->bodyStream);
        if (c->capStream) cudaStreamDestroy(c->capStream);
        dev_free(c->incScratch);
        dev_free(c->sortScratch);
        dev_free(c->block);
        delete c;
        return cuda_fail(e, "context init");
    }
    *out = c;
    return DEM_OK;
}

extern "C" int dem_destroy(DemContext* c) {
    if (!c) return DEM_OK;
    drop_graphs(c);
    drop_profile(c);
    drop_tune_events(c);
    if (c->capStream) cudaStreamDestroy(c->capStream);
    if (c->bodyStream) cudaStreamDestroy(c->bodyStream);
    if (c->forkStream) cudaStreamDestroy(c->forkStream);
    if (c->loopStream) cudaStreamDestroy(c->loopStream);
    if (c->forkEv) cudaEventDestroy(c->forkEv);
    if (c->moverJoinEv) cudaEventDestroy(c->moverJoinEv);
    if (c->moverForkEv) cudaEventDestroy(c->moverForkEv);
    if (c->moverStream) cudaStreamDestroy(c->moverStream);
    if (c->joinEv) cudaEventDestroy(c->joinEv);
    dev_free(c->followRows);
    dev_free(c->followIds);
    dev_free(c->followRing);
    dev_free(c->adjCheck);
    dev_free(c->adjRec);
    dev_free(c->adjTmp);
    dev_free(c->dResBins);
    dev_free(c->dResEntries);
    dev_free(c->resQueue);
    dev_free(c->resWork);
    dev_free(c->clusterWork);
    dev_free(c->renderOwner);
    dev_free(c->ctlBlock);
    dev_free(c->dTable);
    dev_free(c->spec);
    dev_free(c->incScratch);
    dev_free(c->sortScratch);
    dev_free(c->block);
    delete c;
    return DEM_OK;
}

extern "C" int dem_set_system(DemContext* c, const DemSystem* sys) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    if (c->nspec) return fail(DEM_ERR_INVALID_ARG, "dem_set_system: use dem_batch_create for batches");
    int rc = validate(sys);
    if (rc) return rc;
    if (sys->gridSize[0] != c->sys.gridSize[0] || sys->gridSize[1] != c->sys.gridSize[1])
        return fail(DEM_ERR_INVALID_ARG, "grid size is fixed at dem_create");
    if ((sys->numMaterials > 1) != c->typed)
        return fail(DEM_ERR_INVALID_ARG, "single/multi-material layout is fixed at dem_create");
    c->sys = *sys;
    c->P = scene_kparams(c, c->n);
    set_rmax(c->P, c->rmax);
    drop_graphs(c);
    // keys depend on the box size; recompute them and sort from scratch
    c->keysValid = false;
    c->haveOrder = false;
    return DEM_OK;
}

extern "C" int dem_batch_set_systems(DemContext* c, const DemSystem* specs,
                                     uint32_t numSpecimens, void* stream) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    if (!c->nspec) return fail(DEM_ERR_INVALID_ARG, "not a batch; use dem_set_system");
    if (!specs || numSpecimens != c->nspec)
        return fail(DEM_ERR_INVALID_ARG, "need %u specimens", c->nspec);
    std::vector<KParams> table(c->nspec);
    for (uint32_t s = 0; s < c->nspec; ++s) {
        int rc = validate(&specs[s]);
        if (rc) return rc;
        const KParams& old = c->hTable[s];
        if (specs[s].gridSize[0] != old.gx || specs[s].gridSize[1] != old.gy)
            return fail(DEM_ERR_INVALID_ARG, "specimen %u: grid size is fixed at dem_batch_create", s);
        if (specs[s].numParticles != c->partOff[s + 1] - c->partOff[s])
            return fail(DEM_ERR_INVALID_ARG, "specimen %u: particle count is fixed", s);
        if ((specs[s].numMaterials > 1) != (old.nmat > 1))
            return fail(DEM_ERR_INVALID_ARG, "specimen %u: material layout is fixed", s);
        table[s] = make_kparams(&specs[s], specs[s].numParticles);
        table[s].cellOff = old.cellOff;
        set_rmax(table[s], c->rmax);
        bool attract = false;
        for (uint32_t m = 0; m < table[s].nmat; ++m) attract = attract || table[s].at[m] != 0.0f;
        if (attract && c->P.at[0] == 0.0f)
            return fail(DEM_ERR_INVALID_ARG, "specimen %u: attraction was off at create", s);
    }
    // ordered on the caller's stream after the steps already queued there,
    // which read the table; the source is staged before the call returns
    DEM_TRY_CUDA(cudaMemcpyAsync(c->dTable, table.data(), sizeof(KParams) * c->nspec,
                                 cudaMemcpyHostToDevice, (cudaStream_t)stream),
                 "batch table");
    c->hTable.swap(table);
    // keys depend on the boxes; recompute them and sort from scratch
    c->keysValid = false;
    c->haveOrder = false;
    return DEM_OK;
}

namespace {
// Particle counts a context takes: up to its capacity, a batch exactly its
// capacity.
int check_count(const DemContext* c, uint32_t n) {
    if (n > c->capacity) return fail(DEM_ERR_CAPACITY, "n %u > capacity %u", n, c->capacity);
    if (c->nspec && n != c->capacity)
        return fail(DEM_ERR_INVALID_ARG, "a batch takes all %u particles, specimen by specimen",
                    c->capacity);
    return DEM_OK;
}

bool has_state_sets(const DemContext* c) { return c->dyn[0].pos != nullptr; }

// A new state of n particles is in the current sets (set c->cur, positions
// in dyn[0].pos): clears the error word, reads the largest radius back and
// keeps or drops the captured graphs.
int accept_state(DemContext* c, uint32_t n, cudaStream_t st) {
    c->inSortOrder = false;
    // the new state replaces the one any recorded error was about
    DEM_TRY_CUDA(cudaMemsetAsync(c->errFlag, 0, 4, st), "clear error word");
    const int a = c->cur;
    // the largest radius bounds every contact distance (neighbour culling)
    uint32_t rbits = 0;
    DEM_TRY_CUDA(launch_max_radius(c->stat[a].radius, n, c->errFlag + 1, st), "max radius");
    DEM_TRY_CUDA(cudaMemcpyAsync(&rbits, c->errFlag + 1, 4, cudaMemcpyDeviceToHost, st),
                 "max radius copy");
    DEM_TRY_CUDA(cudaStreamSynchronize(st), "set_state sync");
    float rmax;
    memcpy(&rmax, &rbits, 4);
    rmax = (n > 0 && std::isfinite(rmax)) ? rmax : INFINITY;
    // the same particle count and largest radius give the same kernel
    // parameters (and specimen table), so the captured graphs stay valid;
    // only the first step's full sort is forced, as after every new state
    if (n == c->n && n > 0 && memcmp(&rmax, &c->rmax, sizeof(float)) == 0) {
        c->keysValid = false;
        c->haveOrder = false;
        return DEM_OK;
    }
    c->n = n;
    c->rmax = rmax;
    if (c->nspec) {
        for (uint32_t sp = 0; sp < c->nspec; ++sp) set_rmax(c->hTable[sp], c->rmax);
        set_rmax(c->P, c->rmax);
        DEM_TRY_CUDA(cudaMemcpy(c->dTable, c->hTable.data(), sizeof(KParams) * c->nspec,
                                cudaMemcpyHostToDevice),
                     "specimen table");
    } else {
        c->P = scene_kparams(c, n);
        set_rmax(c->P, c->rmax);
    }
    drop_graphs(c);
    c->keysValid = false;
    c->haveOrder = false;
    return DEM_OK;
}
}  // namespace

extern "C" int dem_set_state(DemContext* c, uint32_t n, const float* pos, const float* vel,
                             const float* theta, const float* omega, const float* radius,
                             const float* mass, const uint32_t* id, const uint32_t* type, int host,
                             void* stream) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    int rc = check_count(c, n);
    if (rc) return rc;
    if (!has_state_sets(c))
        return fail(DEM_ERR_INVALID_ARG, "no state buffers: call dem_adopt_state first");
    if (n && (!pos || !vel || !theta || !omega || !radius || !mass || !id))
        return fail(DEM_ERR_INVALID_ARG, "dem_set_state: NULL buffer");
    if (c->typed && n && !type)
        return fail(DEM_ERR_INVALID_ARG, "type array required with more than one material");
    cudaStream_t st = (cudaStream_t)stream;
    const cudaMemcpyKind k = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const int a = c->cur;
    DEM_TRY_CUDA(cudaMemcpyAsync(c->dyn[0].pos, pos, 8ull * n, k, st), "set pos");
    DEM_TRY_CUDA(cudaMemcpyAsync(c->dyn[a].vel, vel, 8ull * n, k, st), "set vel");
    DEM_TRY_CUDA(cudaMemcpyAsync(c->dyn[a].theta, theta, 4ull * n, k, st), "set theta");
    DEM_TRY_CUDA(cudaMemcpyAsync(c->dyn[a].omega, omega, 4ull * n, k, st), "set omega");
    DEM_TRY_CUDA(cudaMemcpyAsync(c->stat[a].radius, radius, 4ull * n, k, st), "set radius");
    DEM_TRY_CUDA(cudaMemcpyAsync(c->stat[a].mass, mass, 4ull * n, k, st), "set mass");
    DEM_TRY_CUDA(cudaMemcpyAsync(c->stat[a].id, id, 4ull * n, k, st), "set id");
    if (c->typed)
        DEM_TRY_CUDA(cudaMemcpyAsync(c->stat[a].type, type, 4ull * n, k, st), "set type");
    return accept_state(c, n, st);
}

static_assert(DEM_STATE_PAD == kFilterPad, "adopted sets carry the step kernel's read padding");

extern "C" int dem_adopt_state(DemContext* c, uint32_t n, const DemStateSet* first,
                               const DemStateSet* second, void* stream) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    int rc = check_count(c, n);
    if (rc) return rc;
    if (n == 0) return fail(DEM_ERR_INVALID_ARG, "dem_adopt_state: n must be > 0");
    if (!first || !second) return fail(DEM_ERR_INVALID_ARG, "dem_adopt_state: NULL set");
    // every array of both sets: its address, its length in bytes and its
    // alignment; they must be present, aligned and pairwise disjoint
    struct Span { const void* p; size_t bytes; size_t align; const char* what; };
    std::vector<Span> spans;
    const DemStateSet* sets[2] = {first, second};
    for (int s = 0; s < 2; ++s) {
        const DemStateSet& d = *sets[s];
        spans.push_back({d.pos, 8ull * (n + DEM_STATE_PAD), 8, "pos"});
        spans.push_back({d.vel, 8ull * n, 8, "vel"});
        spans.push_back({d.theta, 4ull * n, 4, "theta"});
        spans.push_back({d.omega, 4ull * n, 4, "omega"});
        spans.push_back({d.radius, 4ull * (n + DEM_STATE_PAD), 4, "radius"});
        spans.push_back({d.mass, 4ull * n, 4, "mass"});
        spans.push_back({d.id, 4ull * n, 4, "id"});
        if (c->typed) spans.push_back({d.type, 4ull * n, 4, "type"});
    }
    for (const Span& x : spans) {
        if (!x.p) return fail(DEM_ERR_INVALID_ARG, "dem_adopt_state: NULL %s", x.what);
        if (misaligned(x.p, x.align))
            return fail(DEM_ERR_INVALID_ARG, "dem_adopt_state: %s is not %zu-byte aligned", x.what,
                        x.align);
    }
    for (size_t i = 0; i < spans.size(); ++i)
        for (size_t j = i + 1; j < spans.size(); ++j) {
            const uintptr_t a0 = (uintptr_t)spans[i].p, b0 = (uintptr_t)spans[j].p;
            if (a0 < b0 + spans[j].bytes && b0 < a0 + spans[i].bytes)
                return fail(DEM_ERR_INVALID_ARG, "dem_adopt_state: %s of set %zu overlaps %s of set %zu",
                            spans[i].what, i / (spans.size() / 2), spans[j].what,
                            j / (spans.size() / 2));
        }
    for (const Span& x : spans) {
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, x.p) != cudaSuccess || at.type != cudaMemoryTypeDevice ||
            at.device != c->device) {
            cudaGetLastError();
            return fail(DEM_ERR_INVALID_ARG, "dem_adopt_state: %s is not device memory of device %d",
                        x.what, c->device);
        }
    }
    DynSet dyn[2];
    StatSet stat[2];
    for (int s = 0; s < 2; ++s) {
        const DemStateSet& d = *sets[s];
        dyn[s].pos = reinterpret_cast<float2*>(d.pos);
        dyn[s].vel = reinterpret_cast<float2*>(d.vel);
        dyn[s].theta = d.theta;
        dyn[s].omega = d.omega;
        stat[s].radius = d.radius;
        stat[s].mass = d.mass;
        stat[s].id = d.id;
        stat[s].type = c->typed ? d.type : nullptr;
    }
    // the captured graphs hold the buffers' addresses
    if (memcmp(dyn, c->dyn, sizeof(dyn)) != 0 || memcmp(stat, c->stat, sizeof(stat)) != 0)
        drop_graphs(c);
    memcpy(c->dyn, dyn, sizeof(dyn));
    memcpy(c->stat, stat, sizeof(stat));
    c->cur = 0;
    return accept_state(c, n, (cudaStream_t)stream);
}

extern "C" int dem_state_view(DemContext* c, DemStateSet* out, int* setIndex) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    if (!out) return fail(DEM_ERR_INVALID_ARG, "dem_state_view: NULL output");
    if (!has_state_sets(c))
        return fail(DEM_ERR_INVALID_ARG, "no state buffers: call dem_adopt_state first");
    const int a = c->cur;
    out->pos = reinterpret_cast<float*>(c->dyn[0].pos);
    out->vel = reinterpret_cast<float*>(c->dyn[a].vel);
    out->theta = c->dyn[a].theta;
    out->omega = c->dyn[a].omega;
    out->radius = c->stat[a].radius;
    out->mass = c->stat[a].mass;
    out->id = c->stat[a].id;
    out->type = c->typed ? c->stat[a].type : nullptr;
    if (setIndex) *setIndex = a;
    return DEM_OK;
}

extern "C" int dem_get_state(DemContext* c, float* pos, float* vel, float* theta, float* omega,
                             float* radius, float* mass, uint32_t* id, uint32_t* type,
                             uint32_t* loc, float* pressure, float* acc, float* alpha, int host,
                             void* stream) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    if (!has_state_sets(c))
        return fail(DEM_ERR_INVALID_ARG, "no state buffers: call dem_adopt_state first");
    cudaStream_t st = (cudaStream_t)stream;
    const cudaMemcpyKind k = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    const uint32_t n = c->n;
    const int a = c->cur;
    if (pos) DEM_TRY_CUDA(cudaMemcpyAsync(pos, c->dyn[0].pos, 8ull * n, k, st), "get pos");
    if (vel) DEM_TRY_CUDA(cudaMemcpyAsync(vel, c->dyn[a].vel, 8ull * n, k, st), "get vel");
    if (theta) DEM_TRY_CUDA(cudaMemcpyAsync(theta, c->dyn[a].theta, 4ull * n, k, st), "get theta");
    if (omega) DEM_TRY_CUDA(cudaMemcpyAsync(omega, c->dyn[a].omega, 4ull * n, k, st), "get omega");
    if (radius) DEM_TRY_CUDA(cudaMemcpyAsync(radius, c->stat[a].radius, 4ull * n, k, st), "get radius");
    if (mass) DEM_TRY_CUDA(cudaMemcpyAsync(mass, c->stat[a].mass, 4ull * n, k, st), "get mass");
    if (id) DEM_TRY_CUDA(cudaMemcpyAsync(id, c->stat[a].id, 4ull * n, k, st), "get id");
    if (type && c->typed)
        DEM_TRY_CUDA(cudaMemcpyAsync(type, c->stat[a].type, 4ull * n, k, st), "get type");
    if (loc) DEM_TRY_CUDA(cudaMemcpyAsync(loc, c->loc, 4ull * n, k, st), "get loc");
    if (pressure) DEM_TRY_CUDA(cudaMemcpyAsync(pressure, c->pressure, 4ull * n, k, st), "get pressure");
    if (acc) DEM_TRY_CUDA(cudaMemcpyAsync(acc, c->acc, 8ull * n, k, st), "get acc");
    if (alpha) DEM_TRY_CUDA(cudaMemcpyAsync(alpha, c->alpha, 4ull * n, k, st), "get alpha");
    return DEM_OK;
}

// DEM_CTX_DIRECT: the same kernels launched one by one, the sort path
// (incremental, or full after a mover overflow) read back on the host each
// step instead of chosen on the device by conditional graph nodes, so that
// per-kernel profilers see every launch.
int step_direct(DemContext* c, uint32_t nsteps, cudaStream_t st) {
    for (uint32_t s = 0; s < nsteps; ++s) {
        const int a = c->cur;
        bool full = !c->haveOrder;
        if (!full) {
            uint32_t need = 0;
            DEM_TRY_CUDA(cudaMemcpyAsync(&need, c->inc.ctrl + kCtrlNeedFull, 4,
                                         cudaMemcpyDeviceToHost, st),
                         "read sort path");
            DEM_TRY_CUDA(cudaStreamSynchronize(st), "sync");
            full = need != 0u;
        }
        const bool prof = c->profiling && c->evUsed + 3 <= c->evCap;
        cudaEvent_t* ev = prof ? c->evPool + c->evUsed : nullptr;
        if (prof) DEM_TRY_CUDA(cudaEventRecord(ev[0], st), "profile event");
        DEM_TRY_CUDA(full ? enqueue_full_sort(c, a, st, nullptr) : enqueue_inc_sort(c, a, st, nullptr),
                     "sort phase");
        if (prof) DEM_TRY_CUDA(cudaEventRecord(ev[1], st), "profile event");
        if (c->tuned < 0) {
            int rc = tune_prepare(c, false);
            if (rc) return rc;
            const uint32_t k = c->tuneStep;
            const int keep = c->variant;
            c->variant = (int)(k % kStepVariants);
            DEM_TRY_CUDA(cudaEventRecord(c->tuneEv[2 * k], st), "tuner event");
            cudaError_t e = enqueue_step_kernel(c, st, nullptr);
            c->variant = keep;
            DEM_TRY_CUDA(e, "step kernel");
            DEM_TRY_CUDA(cudaEventRecord(c->tuneEv[2 * k + 1], st), "tuner event");
            if (++c->tuneStep == kTuneSteps) {
                rc = tune_finish(c, false);
                if (rc) return rc;
            }
        } else {
            DEM_TRY_CUDA(enqueue_step_kernel(c, st, nullptr), "step kernel");
        }
        if (prof) {
            DEM_TRY_CUDA(cudaEventRecord(ev[2], st), "profile event");
            c->evUsed += 3;
            ++c->stepsProfiled;
        }
        c->cur ^= 1;
        c->haveOrder = true;
        c->inSortOrder = true;
    }
    return DEM_OK;
}

namespace {

bool has_attraction_host(const KParams& P);

constexpr int kNotResident = -1;

// A multi-step call of a batch created with DEM_CTX_RESIDENT as one
// persistent launch (dem_resident.cu).  Returns kNotResident, having done
// nothing, when the batch has types, attraction, a control particle, stage
// profiling or a specimen too large for one bin: the graph path steps it.
// After the launch the state is in the order of its last sort, as after the
// graph path, but no mover record exists: the next graph-path step sorts
// from scratch (the same permutation, the sort being stable).
int resident_step(DemContext* c, uint32_t nsteps, cudaStream_t st) {
    if (c->typed || c->ctlOn || c->profiling || !has_state_sets(c) ||
        c->partOff.size() != (size_t)c->nspec + 1 || c->partOff.back() != c->n)
        return kNotResident;
    for (uint32_t s = 0; s < c->nspec; ++s)
        if (has_attraction_host(c->hTable[s])) return kNotResident;
    if (!c->resPlanned) {
        std::vector<uint32_t> cells(c->nspec);
        for (uint32_t s = 0; s < c->nspec; ++s) cells[s] = c->hTable[s].gx * c->hTable[s].gy;
        std::vector<ResEntry> entries;
        std::vector<ResBin> bins;
        uint32_t maxN = 0, maxC = 0;
        c->resPlanned = true;
        if (!resident_plan(c->partOff, cells, entries, bins, maxN, maxC) || bins.empty()) {
            c->resBins = 0;
            return kNotResident;
        }
        const int blocks = resident_blocks((uint32_t)bins.size(), c->device);
        DEM_TRY_CUDA(dev_alloc(&c->dResBins, sizeof(ResBin) * bins.size()), "cudaMalloc bins");
        DEM_TRY_CUDA(dev_alloc(&c->dResEntries, sizeof(ResEntry) * entries.size()),
                     "cudaMalloc bin entries");
        DEM_TRY_CUDA(dev_alloc(&c->resQueue, sizeof(uint32_t)), "cudaMalloc bin queue");
        DEM_TRY_CUDA(dev_alloc(&c->resWork, resident_work_bytes(maxN) * (size_t)blocks),
                     "cudaMalloc resident scratch");
        DEM_TRY_CUDA(cudaMemcpyAsync(c->dResBins, bins.data(), sizeof(ResBin) * bins.size(),
                                     cudaMemcpyHostToDevice, st),
                     "bins");
        DEM_TRY_CUDA(cudaMemcpyAsync(c->dResEntries, entries.data(),
                                     sizeof(ResEntry) * entries.size(), cudaMemcpyHostToDevice, st),
                     "bin entries");
        DEM_TRY_CUDA(cudaStreamSynchronize(st), "bins");
        c->resBins = (uint32_t)bins.size();
        c->resMaxN = maxN;
        c->resMaxC = maxC;
        c->resBlocks = blocks;
    }
    if (c->resBins == 0) return kNotResident;
    const int a = c->cur;
    ResIO io{c->dyn[0].pos, c->dyn[a].vel, c->dyn[a].theta, c->dyn[a].omega, c->stat[a].radius,
             c->stat[a].mass, c->stat[a].id, c->loc, c->pressure, c->acc, c->alpha};
    DEM_TRY_CUDA(launch_resident(c->dTable, c->dResBins, c->resBins, c->dResEntries, c->resMaxN,
                                 c->resMaxC, c->resQueue, c->resWork, c->resBlocks, io, c->n,
                                 nsteps, c->errFlag, st),
                 "resident step");
    c->keysValid = false;
    c->haveOrder = false;
    c->inSortOrder = false;
    return DEM_OK;
}

// A multi-step call of a single scene created with DEM_CTX_RESIDENT as one
// cluster launch (dem_resident.cu): every block of the cluster holds the
// whole scene in shared memory and steps its share of the slots.  Returns
// kNotResident, having done nothing, for scenes it does not take (more than
// 8,192 disks or cells, types, attraction, a control particle, profiling) or
// when no such cluster can be resident on this GPU; the graph path steps
// those.  The next graph-path step sorts from scratch.
int cluster_step(DemContext* c, uint32_t nsteps, cudaStream_t st) {
    if (c->typed || c->ctlOn || c->profiling || c->clusterUnsupported || c->rows ||
        !has_state_sets(c) ||
        has_attraction_host(c->P) || !cluster_scene_fits(c->n, c->numCells))
        return kNotResident;
    const size_t bytes = cluster_scene_work_bytes(c->n);
    if (c->clusterWorkBytes < bytes) {
        dev_free(c->clusterWork);
        c->clusterWork = nullptr;
        c->clusterWorkBytes = 0;
        DEM_TRY_CUDA(dev_alloc(&c->clusterWork, bytes), "cudaMalloc cluster scratch");
        c->clusterWorkBytes = bytes;
    }
    const int a = c->cur;
    ResIO io{c->dyn[0].pos, c->dyn[a].vel, c->dyn[a].theta, c->dyn[a].omega, c->stat[a].radius,
             c->stat[a].mass, c->stat[a].id, c->loc, c->pressure, c->acc, c->alpha};
    const cudaError_t e = launch_cluster_scene(c->P, c->n, c->numCells, c->clusterWork, io,
                                               nsteps, c->errFlag, st);
    if (e == cudaErrorNotSupported) {
        c->clusterUnsupported = true;
        return kNotResident;
    }
    DEM_TRY_CUDA(e, "cluster step");
    c->keysValid = false;
    c->haveOrder = false;
    c->inSortOrder = false;
    return DEM_OK;
}

}  // namespace

namespace {
int step_graph_path(DemContext* c, uint32_t nsteps, cudaStream_t st);
}  // namespace

extern "C" int dem_step(DemContext* c, uint32_t nsteps, void* stream) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    if (nsteps == 0 || c->n == 0) return DEM_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (c->flags & DEM_CTX_RESIDENT) {
        int rc = c->nspec ? resident_step(c, nsteps, st) : cluster_step(c, nsteps, st);
        if (rc != kNotResident) return rc;
    }
    return step_graph_path(c, nsteps, st);
}

namespace {
// dem_step on the graph path: the sort and step graphs, or the device-side
// step loop for pairs of steps (also the steps of dem_step_followed, whose
// per-step rows are gathered from this path's buffers).
int step_graph_path(DemContext* c, uint32_t nsteps, cudaStream_t st) {
    if (!c->keysValid) {
        if (c->nspec)
            DEM_TRY_CUDA(launch_calc_hash_batched(c->dTable, c->spec, c->dyn[0].pos, c->keys, c->n,
                                                  st),
                         "hash");
        else
            DEM_TRY_CUDA(launch_calc_hash(c->P, c->dyn[0].pos, c->keys, nullptr, c->n, st),
                         "hash");
        c->keysValid = true;
        c->haveOrder = false;
    }
    if (c->flags & DEM_CTX_DIRECT) return step_direct(c, nsteps, st);
    for (int p = 0; p < 2; ++p) {
        for (int k = 0; k < 2; ++k)
            if (!c->sortGraph[k][p]) {
                int rc = build_graph(c, k, p);
                if (rc) return rc;
            }
        if (!c->stepGraph[p]) {
            int rc = build_graph(c, 2, p);
            if (rc) return rc;
        }
    }
    for (uint32_t s = 0; s < nsteps; ++s) {
        // Pairs of steps run inside the device-side loop, one graph launch for
        // all of them, unless the host has work between steps (stage
        // profiling, the tuner) or there is no previous order yet (the first
        // sort is a full sort).
        if (!c->profiling && c->tuned >= 0 && c->haveOrder && nsteps - s >= 2) {
            const uint32_t pairs = (nsteps - s) / 2;
            const int p = c->cur;
            if (!c->loopGraph[p]) {
                int rc = build_loop_graph(c, p);
                if (rc) return rc;
            }
            DEM_TRY_CUDA(launch_set_words(c->loopCtl + kLoopStepReq, Words{{pairs}, 1u}, st),
                         "step loop count");
            DEM_TRY_CUDA(cudaGraphLaunch(c->loopGraph[p], st), "graph launch");
            s += 2 * pairs - 1;  // an even number of steps leaves the parity as it was
            continue;
        }
        const int p = c->cur;
        const int kind = c->haveOrder ? 1 : 0;
        const bool prof = c->profiling && c->evUsed + 3 <= c->evCap;
        cudaEvent_t* ev = prof ? c->evPool + c->evUsed : nullptr;
        if (prof) DEM_TRY_CUDA(cudaEventRecord(ev[0], st), "profile event");
        DEM_TRY_CUDA(cudaGraphLaunch(c->sortGraph[kind][p], st), "graph launch");
        if (prof) DEM_TRY_CUDA(cudaEventRecord(ev[1], st), "profile event");
        if (c->tuned < 0) {
            int rc = tune_prepare(c, true);
            if (rc) return rc;
            const uint32_t k = c->tuneStep;
            DEM_TRY_CUDA(cudaEventRecord(c->tuneEv[2 * k], st), "tuner event");
            DEM_TRY_CUDA(cudaGraphLaunch(c->tuneGraph[k % kStepVariants][p], st), "graph launch");
            DEM_TRY_CUDA(cudaEventRecord(c->tuneEv[2 * k + 1], st), "tuner event");
            if (++c->tuneStep == kTuneSteps) {
                rc = tune_finish(c, true);
                if (rc) return rc;
            }
        } else {
            DEM_TRY_CUDA(cudaGraphLaunch(c->stepGraph[p], st), "graph launch");
        }
        if (prof) {
            DEM_TRY_CUDA(cudaEventRecord(ev[2], st), "profile event");
            c->evUsed += 3;
            ++c->stepsProfiled;
        }
        c->cur ^= 1;
        c->haveOrder = true;
        c->inSortOrder = true;
    }
    return DEM_OK;
}
}  // namespace

extern "C" int dem_set_step_variant(DemContext* c, int32_t variant) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    if (variant < 0 || variant >= kStepVariants)
        return fail(DEM_ERR_INVALID_ARG, "step variant %d outside 0..%d", (int)variant,
                    kStepVariants - 1);
    drop_tune_graphs(c);
    drop_tune_events(c);
    c->tuneStep = 0;
    c->tuned = 0;
    if (c->variant != variant) {
        c->variant = variant;
        for (int p = 0; p < 2; ++p) {
            if (c->stepGraph[p]) cudaGraphExecDestroy(c->stepGraph[p]);
            c->stepGraph[p] = nullptr;
        }
        drop_loop_graphs(c);
    }
    return DEM_OK;
}

extern "C" int dem_get_step_variant(DemContext* c, DemStepVariant* out) {
    if (!c || !out) return fail(DEM_ERR_INVALID_ARG, "context or out is NULL");
    const StepShape sh = step_variant_shape(c->ctlOn ? 0 : c->variant);
    out->variant = c->variant;
    out->threads = (uint32_t)sh.threads;
    out->blocksPerSm = (uint32_t)sh.blocksPerSm;
    out->tuned = c->tuned;
    for (int v = 0; v < DEM_STEP_VARIANTS; ++v) out->medianMs[v] = c->tuned > 0 ? c->tuneMs[v] : 0.0f;
    return DEM_OK;
}

extern "C" int dem_get_cells(DemContext* c, uint32_t* cellStart, uint32_t* cellEnd,
                             void* stream) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    DEM_TRY_CUDA(launch_unpack_cells(c->cells[c->cur], c->numCells, cellStart, cellEnd,
                                     (cudaStream_t)stream),
                 "unpack cells");
    return DEM_OK;
}

extern "C" int dem_row_slots(DemContext* c, uint32_t rowLo, uint32_t rowHi, uint32_t* first,
                             uint32_t* count, void* stream) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    if (c->nspec) return fail(DEM_ERR_INVALID_ARG, "dem_row_slots takes a single scene");
    if (!first || !count) return fail(DEM_ERR_INVALID_ARG, "dem_row_slots: NULL output");
    // the scene's rows; a row window holds rows [rowFirst, rowFirst + rows),
    // of which those past the grid's last row do not exist
    const uint32_t gx = c->sys.gridSize[0], gy = c->sys.gridSize[1];
    const uint32_t lo0 = c->rowFirst, hi0 = std::min(c->rowFirst + (c->rows ? c->rows : gy), gy);
    if (rowLo > rowHi || rowLo < lo0 || rowHi > hi0)
        return fail(DEM_ERR_INVALID_ARG, "rows [%u, %u) outside the context's rows [%u, %u)",
                    rowLo, rowHi, lo0, hi0);
    rowLo -= lo0;
    rowHi -= lo0;
    if (!c->inSortOrder)
        return fail(DEM_ERR_INVALID_ARG, "the state is not in the order of a sort: step first");
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t* f = c->first[c->cur];
    uint32_t w[2];
    DEM_TRY_CUDA(cudaMemcpyAsync(&w[0], f + (size_t)rowLo * gx, 4, cudaMemcpyDeviceToHost, st),
                 "row slots");
    DEM_TRY_CUDA(cudaMemcpyAsync(&w[1], f + (size_t)rowHi * gx, 4, cudaMemcpyDeviceToHost, st),
                 "row slots");
    DEM_TRY_CUDA(cudaStreamSynchronize(st), "row slots sync");
    *first = w[0];
    *count = w[1] - w[0];
    return DEM_OK;
}

extern "C" int dem_check(DemContext* c, void* stream) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    uint32_t flag = 0;
    cudaStream_t st = (cudaStream_t)stream;
    DEM_TRY_CUDA(cudaMemcpyAsync(&flag, c->errFlag, 4, cudaMemcpyDeviceToHost, st), "read flag");
    DEM_TRY_CUDA(cudaStreamSynchronize(st), "sync");
    if (flag & kSortTimeoutBit)
        return fail(DEM_ERR_TIMEOUT, "a bounded wait in the sort gave up; the state is invalid");
    if (flag) return fail(DEM_ERR_OOB, "a particle position became NaN or infinite");
    return DEM_OK;
}

extern "C" int dem_debug_fail_allocation(int nth) {
    if (nth < 0) return fail(DEM_ERR_INVALID_ARG, "nth must be >= 0");
    g_failCountdown.store(nth);
    return DEM_OK;
}

extern "C" long long dem_debug_live_allocations(void) { return g_liveAllocs.load(); }

extern "C" int dem_debug_sort_hold(DemContext* c, uint32_t holdTile, uint32_t spinLimit) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    c->ss.holdTile = holdTile;
    c->ss.spinLimit = spinLimit ? spinLimit : kSortSpinLimit;
    drop_graphs(c);  // the sort's kernels take both as launch parameters
    return DEM_OK;
}

extern "C" int dem_kernels_per_step(DemContext* c) {
    if (!c) return -1;
    if (!c->sortGraph[1][0] && c->n > 0) {
        if (build_graph(c, 1, 0) != DEM_OK) return -1;
    }
    return c->launchesPerStep;
}

namespace {
int get_followed(DemContext* c, const uint32_t* ids, uint32_t count, float* rows, void* stream,
                 bool sync) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    if (count == 0) return DEM_OK;
    if (!ids || !rows) return fail(DEM_ERR_INVALID_ARG, "dem_get_followed: NULL buffer");
    for (uint32_t i = 0; i < count; ++i)
        if (ids[i] >= c->n) return fail(DEM_ERR_INVALID_ARG, "followed id %u >= n %u", ids[i], c->n);
    if (!c->followRows) {
        DEM_TRY_CUDA(dev_alloc(&c->followRows, sizeof(float) * 12 * kFollowBatch),
                     "cudaMalloc followed rows");
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int a = c->cur;
    for (uint32_t base = 0; base < count; base += kFollowBatch) {
        FollowIds f;
        f.count = count - base < kFollowBatch ? count - base : kFollowBatch;
        for (uint32_t i = 0; i < f.count; ++i) f.id[i] = ids[base + i];
        DEM_TRY_CUDA(launch_followed(f, c->loc, state_dyn(c), c->stat[a],
                                     (c->flags & DEM_CTX_ACCEL) ? c->acc : nullptr,
                                     (c->flags & DEM_CTX_ACCEL) ? c->alpha : nullptr,
                                     (c->flags & DEM_CTX_PRESSURE) ? c->pressure : nullptr,
                                     c->followRows, st),
                     "followed gather");
        DEM_TRY_CUDA(cudaMemcpyAsync(rows + 12ull * base, c->followRows,
                                     sizeof(float) * 12 * f.count, cudaMemcpyDefault, st),
                     "followed copy");
        // the staging buffer is reused by the next batch of ids
        if (sync || base + kFollowBatch < count)
            DEM_TRY_CUDA(cudaStreamSynchronize(st), "followed sync");
    }
    return DEM_OK;
}
}  // namespace

extern "C" int dem_get_followed(DemContext* c, const uint32_t* ids, uint32_t count, float* rows,
                                void* stream) {
    return get_followed(c, ids, count, rows, stream, true);
}

extern "C" int dem_get_followed_async(DemContext* c, const uint32_t* ids, uint32_t count,
                                      float* rows, void* stream) {
    return get_followed(c, ids, count, rows, stream, false);
}

namespace {
constexpr size_t kFollowRingBytes = 64ull << 20;  // rows of one chunk of steps
}  // namespace

extern "C" int dem_step_followed(DemContext* c, uint32_t nsteps, const uint32_t* ids,
                                 uint32_t count, float* rows, void* stream) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    if (count == 0 || nsteps == 0) return dem_step(c, nsteps, stream);
    if (!ids || !rows) return fail(DEM_ERR_INVALID_ARG, "dem_step_followed: NULL buffer");
    for (uint32_t i = 0; i < count; ++i)
        if (ids[i] >= c->n) return fail(DEM_ERR_INVALID_ARG, "followed id %u >= n %u", ids[i], c->n);
    cudaStream_t st = (cudaStream_t)stream;
    const size_t rowBytes = 48ull * count;  // one step's rows
    const uint32_t chunk =
        (uint32_t)std::min<size_t>(nsteps, std::max<size_t>(1, kFollowRingBytes / rowBytes));
    if (c->followIdsCap < count) {
        drop_loop_graphs(c);
        dev_free(c->followIds);
        c->followIds = nullptr;
        c->followIdsCap = 0;
        DEM_TRY_CUDA(dev_alloc(&c->followIds, 4ull * count), "cudaMalloc followed ids");
        c->followIdsCap = count;
    }
    if (c->followRingBytes < chunk * rowBytes) {
        drop_loop_graphs(c);
        dev_free(c->followRing);
        c->followRing = nullptr;
        c->followRingBytes = 0;
        DEM_TRY_CUDA(dev_alloc(&c->followRing, chunk * rowBytes), "cudaMalloc followed rows");
        c->followRingBytes = chunk * rowBytes;
    }
    // the ids go through a library-owned host copy, so they are read before
    // this call returns whatever memory the caller passed
    c->followIdsHost.assign(ids, ids + count);
    DEM_TRY_CUDA(cudaMemcpyAsync(c->followIds, c->followIdsHost.data(), 4ull * count,
                                 cudaMemcpyHostToDevice, st),
                 "followed ids");
    DEM_TRY_CUDA(launch_set_words(c->loopCtl + kLoopFolCount, Words{{count}, 1u}, st),
                 "followed count");
    for (uint32_t s = 0; s < nsteps;) {
        const uint32_t m = std::min(chunk, nsteps - s);
        for (uint32_t j = 0; j < m;) {
            // pairs of steps with their rows in the device-side loop, as in
            // dem_step; a step with host work around it (the first after
            // dem_set_state, tuning, profiling, direct launches) alone
            if (!(c->flags & DEM_CTX_DIRECT) && !c->profiling && c->tuned >= 0 && c->haveOrder &&
                m - j >= 2) {
                const uint32_t pairs = (m - j) / 2;
                const int p = c->cur;
                if (!c->followGraph[p]) {
                    int rc = build_follow_graph(c, p);
                    if (rc) return rc;
                }
                DEM_TRY_CUDA(launch_set_words(c->loopCtl + kLoopFolReq, Words{{pairs, 0u, j}, 3u}, st),
                             "followed loop count");
                DEM_TRY_CUDA(cudaGraphLaunch(c->followGraph[p], st), "graph launch");
                j += 2 * pairs;
            } else {
                // the graph path: the rows are gathered from its buffers
                int rc = step_graph_path(c, 1, st);
                if (rc) return rc;
                DEM_TRY_CUDA(enqueue_followed_ring(c, c->cur ^ 1, nullptr, j, st), "followed gather");
                ++j;
            }
        }
        DEM_TRY_CUDA(cudaMemcpyAsync(rows + (size_t)s * count * 12, c->followRing, m * rowBytes,
                                     cudaMemcpyDefault, st),
                     "followed rows copy");
        s += m;
    }
    return DEM_OK;
}

namespace {
int check_render(const DemRenderParams* rp) {
    if (!rp) return fail(DEM_ERR_INVALID_ARG, "render parameters are NULL");
    if (rp->imageDIMx == 0 || rp->imageDIMy == 0 ||
        (uint64_t)rp->imageDIMx * rp->imageDIMy > (1ull << 30))
        return fail(DEM_ERR_INVALID_ARG, "image %u x %u", rp->imageDIMx, rp->imageDIMy);
    if (rp->colorByPressure && !(rp->maxPressure > 0.0f))
        return fail(DEM_ERR_INVALID_ARG, "maxPressure must be > 0 to colour by pressure");
    return DEM_OK;
}
}  // namespace

extern "C" int dem_render_particles(const DemSystem* sys, const float* pos, const float* theta,
                                    const uint32_t* type, const float* radius,
                                    const float* pressure, uint32_t n, const DemRenderParams* rp,
                                    uint32_t* owner, void* image, void* stream) {
    int rc = validate(sys);
    if (rc) return rc;
    rc = check_render(rp);
    if (rc) return rc;
    if (!owner || !image || (n && (!pos || !radius || (rp->viewRotations && !theta))))
        return fail(DEM_ERR_INVALID_ARG, "dem_render_particles: NULL buffer");
    if (sys->numMaterials > 1 && n && !type)
        return fail(DEM_ERR_INVALID_ARG, "dem_render_particles: several materials need `type`");
    DEM_TRY_CUDA(launch_render(*rp, sys->cubeDimension[0], sys->cubeDimension[1],
                               reinterpret_cast<const float2*>(pos), theta,
                               sys->numMaterials > 1 ? type : nullptr, radius, pressure, n, owner,
                               static_cast<uchar4*>(image), (cudaStream_t)stream),
                 "render");
    return DEM_OK;
}

extern "C" int dem_render(DemContext* c, const DemRenderParams* rp, void* image, void* stream) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    if (c->nspec) return fail(DEM_ERR_INVALID_ARG, "dem_render takes a single scene");
    int rc = check_render(rp);
    if (rc) return rc;
    if (!image) return fail(DEM_ERR_INVALID_ARG, "dem_render: NULL image");
    if (!has_state_sets(c))
        return fail(DEM_ERR_INVALID_ARG, "no state buffers: call dem_adopt_state first");
    const size_t words = (size_t)rp->imageDIMx * rp->imageDIMy;
    if (c->renderOwnerWords < words) {
        dev_free(c->renderOwner);
        c->renderOwner = nullptr;
        c->renderOwnerWords = 0;
        DEM_TRY_CUDA(dev_alloc(&c->renderOwner, 4 * words), "cudaMalloc render scratch");
        c->renderOwnerWords = words;
    }
    const int a = c->cur;
    DEM_TRY_CUDA(launch_render(*rp, c->sys.cubeDimension[0], c->sys.cubeDimension[1],
                               c->dyn[0].pos, c->dyn[a].theta, c->typed ? c->stat[a].type : nullptr,
                               c->stat[a].radius,
                               (c->flags & DEM_CTX_PRESSURE) ? c->pressure : nullptr, c->n,
                               c->renderOwner, static_cast<uchar4*>(image), (cudaStream_t)stream),
                 "render");
    return DEM_OK;
}

extern "C" int dem_set_control(DemContext* c, const DemControl* ctl, void* stream) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    cudaStream_t st = (cudaStream_t)stream;
    if (!ctl) {
        if (c->ctlOn) {
            c->ctlOn = false;
            drop_graphs(c);
        }
        return DEM_OK;
    }
    if (c->nspec) return fail(DEM_ERR_INVALID_ARG, "the control particle takes a single scene");
    if (ctl->material >= c->sys.numMaterials || (!c->typed && ctl->material != 0))
        return fail(DEM_ERR_INVALID_ARG, "control material %u (the context has %u)", ctl->material,
                    c->typed ? c->sys.numMaterials : 1u);
    if (!(ctl->radius > 0.0f) || !std::isfinite(ctl->radius))
        return fail(DEM_ERR_INVALID_ARG, "control radius must be positive and finite");
    if (!c->ctlBlock) {
        const size_t cap = c->capacity ? c->capacity : 1;
        const size_t blocks = (cap + 511) / 512 + 1;
        const size_t bytes = al256(sizeof(ControlDev)) + al256(12 * cap) + al256(12 * blocks) + 256;
        DEM_TRY_CUDA(dev_alloc(&c->ctlBlock, bytes), "cudaMalloc control particle");
        DEM_TRY_CUDA(cudaMemsetAsync(c->ctlBlock, 0, bytes, st), "clear control particle");
        char* q = static_cast<char*>(c->ctlBlock);
        c->dCtl = reinterpret_cast<ControlDev*>(q); q += al256(sizeof(ControlDev));
        c->ctlVec = reinterpret_cast<float*>(q); q += al256(12 * cap);
        c->ctlPartials = reinterpret_cast<float*>(q); q += al256(12 * blocks);
        c->ctlOut = reinterpret_cast<float*>(q);
    }
    ControlDev d;
    d.pos = make_float2(ctl->pos[0], ctl->pos[1]);
    d.vel = make_float2(ctl->vel[0], ctl->vel[1]);
    d.theta = ctl->theta;
    d.omega = ctl->omega;
    d.radius = ctl->radius;
    d.mat = ctl->material;
    d.drift[0] = ctl->drift[0];
    d.drift[1] = ctl->drift[1];
    d.wrapYBelow = ctl->wrapYBelow;
    d.wrapYTo = ctl->wrapYTo;
    d.wrapXAbove = ctl->wrapXAbove;
    d.wrapXTo = ctl->wrapXTo;
    // ordered on the caller's stream after the steps already queued there,
    // which read and move the control particle; the source is staged before
    // the call returns
    DEM_TRY_CUDA(cudaMemcpyAsync(c->dCtl, &d, sizeof(d), cudaMemcpyHostToDevice, st),
                 "set control");
    if (!c->ctlOn) {
        c->ctlOn = true;
        drop_graphs(c);
    }
    return DEM_OK;
}

extern "C" int dem_get_control(DemContext* c, DemControl* ctl, float* reaction, void* stream) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    if (!c->ctlOn) return fail(DEM_ERR_INVALID_ARG, "no control particle");
    cudaStream_t st = (cudaStream_t)stream;
    ControlDev d;
    DEM_TRY_CUDA(cudaMemcpyAsync(&d, c->dCtl, sizeof(d), cudaMemcpyDeviceToHost, st), "get control");
    float r[3] = {0, 0, 0};
    DEM_TRY_CUDA(cudaMemcpyAsync(r, c->ctlOut, sizeof(r), cudaMemcpyDeviceToHost, st), "get reaction");
    DEM_TRY_CUDA(cudaStreamSynchronize(st), "sync");
    if (ctl) {
        ctl->pos[0] = d.pos.x;
        ctl->pos[1] = d.pos.y;
        ctl->vel[0] = d.vel.x;
        ctl->vel[1] = d.vel.y;
        ctl->theta = d.theta;
        ctl->omega = d.omega;
        ctl->radius = d.radius;
        ctl->material = d.mat;
        ctl->drift[0] = d.drift[0];
        ctl->drift[1] = d.drift[1];
        ctl->wrapYBelow = d.wrapYBelow;
        ctl->wrapYTo = d.wrapYTo;
        ctl->wrapXAbove = d.wrapXAbove;
        ctl->wrapXTo = d.wrapXTo;
    }
    if (reaction) memcpy(reaction, r, sizeof(r));
    return DEM_OK;
}

extern "C" int dem_profile_begin(DemContext* c, uint32_t maxSteps) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    if (maxSteps == 0) return fail(DEM_ERR_INVALID_ARG, "maxSteps must be > 0");
    drop_profile(c);
    const uint32_t cap = maxSteps * 3;
    c->evPool = new (std::nothrow) cudaEvent_t[cap];
    if (!c->evPool) return fail(DEM_ERR_NO_MEMORY, "host allocation failed");
    for (uint32_t i = 0; i < cap; ++i) {
        cudaError_t e = cudaEventCreate(&c->evPool[i]);
        if (e != cudaSuccess) {
            c->evCap = i;
            drop_profile(c);
            return cuda_fail(e, "cudaEventCreate");
        }
    }
    c->evCap = cap;
    c->evUsed = 0;
    c->stepsProfiled = 0;
    c->profiling = true;
    return DEM_OK;
}

extern "C" int dem_profile_end(DemContext* c, float* ms, uint32_t* steps) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    if (!c->profiling) return fail(DEM_ERR_INVALID_ARG, "profiling was not started");
    float acc[DEM_NUM_STAGES] = {0.0f, 0.0f, 0.0f};
    if (c->evUsed) DEM_TRY_CUDA(cudaEventSynchronize(c->evPool[c->evUsed - 1]), "event sync");
    for (uint32_t s = 0; s < c->stepsProfiled; ++s) {
        cudaEvent_t* e = c->evPool + 3 * s;
        float t0 = 0.0f, t1 = 0.0f;
        DEM_TRY_CUDA(cudaEventElapsedTime(&t0, e[0], e[1]), "event elapsed");
        DEM_TRY_CUDA(cudaEventElapsedTime(&t1, e[1], e[2]), "event elapsed");
        acc[0] += t0;
        acc[2] += t1;
    }
    if (ms)
        for (int k = 0; k < DEM_NUM_STAGES; ++k) ms[k] = acc[k];
    if (steps) *steps = c->stepsProfiled;
    drop_profile(c);
    return DEM_OK;
}

// ---------------------------------------------------------------------------
// adjoint
// ---------------------------------------------------------------------------
namespace {

size_t snapshot_bytes(uint32_t n) { return al256(8ull * n) * 2 + al256(4ull * n) * 5; }

struct Snapshot {
    float *pos, *vel, *theta, *omega, *radius, *mass;
    uint32_t* id;
};

Snapshot carve_snapshot(void* base, uint32_t n) {
    char* p = static_cast<char*>(base);
    Snapshot s;
    s.pos = reinterpret_cast<float*>(p); p += al256(8ull * n);
    s.vel = reinterpret_cast<float*>(p); p += al256(8ull * n);
    s.theta = reinterpret_cast<float*>(p); p += al256(4ull * n);
    s.omega = reinterpret_cast<float*>(p); p += al256(4ull * n);
    s.radius = reinterpret_cast<float*>(p); p += al256(4ull * n);
    s.mass = reinterpret_cast<float*>(p); p += al256(4ull * n);
    s.id = reinterpret_cast<uint32_t*>(p);
    return s;
}

// One step as dem_step takes it; with `rec`, the sorted state, cell ranges
// and accelerations of the step are copied there.
int step_recorded(DemContext* c, cudaStream_t st, char* rec) {
    const int p = c->cur, b = c->cur ^ 1;
    const int kind = c->haveOrder ? 1 : 0;
    DEM_TRY_CUDA(cudaGraphLaunch(c->sortGraph[kind][p], st), "graph launch");
    DEM_TRY_CUDA(cudaGraphLaunch(c->stepGraph[p], st), "graph launch");
    // the step kernel leaves the sorted state it read intact: record it, the
    // cell ranges and the accelerations in one launch
    if (rec)
        DEM_TRY_CUDA(adj_record_step(rec, RecSlot{}, c->n, c->numCells, step_in(c, p),
                                     step_in_static(c, p),
                                     c->src, c->cells[b],
                                     c->acc, c->alpha, st),
                     "record");
    c->cur ^= 1;
    c->haveOrder = true;
    c->inSortOrder = true;
    return DEM_OK;
}

// dem_set_state from a checkpoint of this context, without its stream
// synchronisation and graph rebuild: a checkpoint holds the same particles,
// so the largest radius, the kernel parameters and the graphs stay valid;
// the next step sorts from scratch.
int restore_checkpoint(DemContext* c, const Snapshot& s, cudaStream_t st) {
    const int a = c->cur;
    const size_t n = c->n;
    DEM_TRY_CUDA(cudaMemcpyAsync(c->dyn[0].pos, s.pos, 8 * n, cudaMemcpyDeviceToDevice, st), "restore pos");
    DEM_TRY_CUDA(cudaMemcpyAsync(c->dyn[a].vel, s.vel, 8 * n, cudaMemcpyDeviceToDevice, st), "restore vel");
    DEM_TRY_CUDA(cudaMemcpyAsync(c->dyn[a].theta, s.theta, 4 * n, cudaMemcpyDeviceToDevice, st), "restore theta");
    DEM_TRY_CUDA(cudaMemcpyAsync(c->dyn[a].omega, s.omega, 4 * n, cudaMemcpyDeviceToDevice, st), "restore omega");
    DEM_TRY_CUDA(cudaMemcpyAsync(c->stat[a].radius, s.radius, 4 * n, cudaMemcpyDeviceToDevice, st), "restore radius");
    DEM_TRY_CUDA(cudaMemcpyAsync(c->stat[a].mass, s.mass, 4 * n, cudaMemcpyDeviceToDevice, st), "restore mass");
    DEM_TRY_CUDA(cudaMemcpyAsync(c->stat[a].id, s.id, 4 * n, cudaMemcpyDeviceToDevice, st), "restore id");
    c->keysValid = false;
    c->haveOrder = false;
    c->inSortOrder = false;
    return DEM_OK;
}

bool has_attraction_host(const KParams& P) {
    for (uint32_t m = 0; m < P.nmat; ++m)
        if (P.at[m] != 0.0f) return true;
    return false;
}

int adj_check_context(DemContext* c) {
    if (!c) return fail(DEM_ERR_INVALID_ARG, "context is NULL");
    if (c->typed) return fail(DEM_ERR_INVALID_ARG, "the adjoint takes a single material");
    if (c->ctlOn) return fail(DEM_ERR_INVALID_ARG, "the adjoint has no control particle");
    if (c->rows) return fail(DEM_ERR_INVALID_ARG, "the adjoint takes a context over the whole grid");
    if (!(c->flags & DEM_CTX_ACCEL)) return fail(DEM_ERR_INVALID_ARG, "create the context with DEM_CTX_ACCEL");
    const uint32_t ns = c->nspec ? c->nspec : 1u;
    for (uint32_t s = 0; s < ns; ++s) {
        const KParams& P = c->nspec ? c->hTable[s] : c->P;
        if (P.gx < 3 || P.gy < 3)
            return fail(DEM_ERR_INVALID_ARG, "the adjoint needs at least 3 cells per axis");
        if (has_attraction_host(P)) return fail(DEM_ERR_INVALID_ARG, "the adjoint has no attraction law");
    }
    return DEM_OK;
}

}  // namespace

extern "C" int dem_adj_forward(DemContext* c, uint32_t nsteps, uint32_t every, void* stream) {
    int rc = adj_check_context(c);
    if (rc) return rc;
    if (nsteps == 0 || every == 0) return fail(DEM_ERR_INVALID_ARG, "nsteps and every must be > 0");
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t windows = (nsteps + every - 1) / every;
    const size_t snap = snapshot_bytes(c->n);
    if (c->adjCheckBytes < snap * windows) {
        dev_free(c->adjCheck);
        c->adjCheck = nullptr;
        c->adjCheckBytes = 0;
        DEM_TRY_CUDA(dev_alloc(&c->adjCheck, snap * windows), "cudaMalloc checkpoints");
        c->adjCheckBytes = snap * windows;
    }
    for (uint32_t w = 0; w < windows; ++w) {
        Snapshot s = carve_snapshot(static_cast<char*>(c->adjCheck) + snap * w, c->n);
        rc = dem_get_state(c, s.pos, s.vel, s.theta, s.omega, s.radius, s.mass, s.id, nullptr,
                           nullptr, nullptr, nullptr, nullptr, 0, stream);
        if (rc) return rc;
        const uint32_t k = std::min(every, nsteps - w * every);
        rc = dem_step(c, k, stream);
        if (rc) return rc;
    }
    DEM_TRY_CUDA(cudaStreamSynchronize(st), "adjoint forward");
    c->adjSteps = nsteps;
    c->adjEvery = every;
    c->adjWindows = windows;
    c->adjN = c->n;
    c->adjRmax = c->rmax;
    return DEM_OK;
}

extern "C" int dem_adj_backward(DemContext* c, float* lamPos, float* lamVel, float* lamOmega,
                                double* grad, void* stream) {
    int rc = adj_check_context(c);
    if (rc) return rc;
    if (!c->adjWindows) return fail(DEM_ERR_INVALID_ARG, "run dem_adj_forward first");
    if (c->n != c->adjN || !(c->rmax == c->adjRmax))
        return fail(DEM_ERR_INVALID_ARG,
                    "the particles changed since dem_adj_forward (dem_set_state): run it again");
    if (!lamPos || !lamVel || !lamOmega || !grad) return fail(DEM_ERR_INVALID_ARG, "NULL buffer");
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t n = c->n;
    const size_t stepBytes = adj_step_bytes(n, c->numCells);
    const uint32_t ns = c->nspec ? c->nspec : 1u;
    const size_t tmpBytes = 2 * al256(8ull * n) + 2 * al256(4ull * n) + al256(8ull * n) +
                            al256(adj_acc_bytes(n)) + al256(8ull * DEM_ADJ_NUM_COEF * ns) +
                            al256(4ull * (ns + 1));
    // the record and scratch persist in the context; a loop captured with
    // other buffers, another record layout or other cotangent buffers is
    // rebuilt
    const size_t recBytes = stepBytes * c->adjEvery;
    if (c->adjRecBytes < recBytes || c->adjTmpBytes < tmpBytes) drop_adj_graphs(c);
    if (c->adjRecBytes < recBytes) {
        dev_free(c->adjRec);
        c->adjRec = nullptr;
        c->adjRecBytes = 0;
        DEM_TRY_CUDA(dev_alloc(&c->adjRec, recBytes), "cudaMalloc adjoint record");
        c->adjRecBytes = recBytes;
    }
    if (c->adjTmpBytes < tmpBytes) {
        dev_free(c->adjTmp);
        c->adjTmp = nullptr;
        c->adjTmpBytes = 0;
        DEM_TRY_CUDA(dev_alloc(&c->adjTmp, tmpBytes), "cudaMalloc adjoint scratch");
        c->adjTmpBytes = tmpBytes;
    }
    if (c->adjRevStepBytes != stepBytes || c->adjRevN != n) drop_adj_graphs(c);
    if (c->adjRevKey[0] != lamPos || c->adjRevKey[1] != lamVel || c->adjRevKey[2] != lamOmega) {
        if (c->adjRevLoop) cudaGraphExecDestroy(c->adjRevLoop);
        c->adjRevLoop = nullptr;
    }
    c->adjRevStepBytes = stepBytes;
    c->adjRevN = n;
    c->adjRevKey[0] = lamPos;
    c->adjRevKey[1] = lamVel;
    c->adjRevKey[2] = lamOmega;
    char* rec = static_cast<char*>(c->adjRec);
    cudaError_t e = cudaSuccess;
    char* q = static_cast<char*>(c->adjTmp);
    float2* tlx = reinterpret_cast<float2*>(q); q += al256(8ull * n);
    float2* tlv = reinterpret_cast<float2*>(q); q += al256(8ull * n);
    float* tlw = reinterpret_cast<float*>(q); q += al256(4ull * n);
    float* lamM = reinterpret_cast<float*>(q); q += al256(4ull * n);
    float2* lamF = reinterpret_cast<float2*>(q); q += al256(8ull * n);
    double* acc = reinterpret_cast<double*>(q); q += al256(adj_acc_bytes(n));
    double* sum = reinterpret_cast<double*>(q); q += al256(8ull * DEM_ADJ_NUM_COEF * ns);
    uint32_t* first = c->nspec ? reinterpret_cast<uint32_t*>(q) : nullptr;
    rc = DEM_OK;
    e = cudaMemsetAsync(acc, 0, adj_acc_bytes(n), st);
    if (e == cudaSuccess && first)
        e = cudaMemcpyAsync(first, c->partOff.data(), 4ull * (ns + 1), cudaMemcpyHostToDevice, st);
    const size_t snap = snapshot_bytes(n);
    cudaGraphExec_t* recLoop = c->adjRecLoop;
    cudaGraphExec_t& revLoop = c->adjRevLoop;
    for (int w = (int)c->adjWindows - 1; w >= 0 && rc == DEM_OK && e == cudaSuccess; --w) {
        rc = restore_checkpoint(c, carve_snapshot(static_cast<char*>(c->adjCheck) + snap * w, n),
                                st);
        if (rc) break;
        const uint32_t k = std::min(c->adjEvery, c->adjSteps - (uint32_t)w * c->adjEvery);
        if (!c->keysValid) {
            e = c->nspec ? launch_calc_hash_batched(c->dTable, c->spec, c->dyn[0].pos, c->keys, n, st)
                         : launch_calc_hash(c->P, c->dyn[0].pos, c->keys, nullptr, n, st);
            c->keysValid = true;
            c->haveOrder = false;
        }
        for (int pp = 0; pp < 2 && rc == DEM_OK; ++pp) {
            for (int kk = 0; kk < 2 && rc == DEM_OK; ++kk)
                if (!c->sortGraph[kk][pp]) rc = build_graph(c, kk, pp);
            if (rc == DEM_OK && !c->stepGraph[pp]) rc = build_graph(c, 2, pp);
        }
        if (rc != DEM_OK || e != cudaSuccess) break;
        // The window's first step sorts from scratch (host-launched, record
        // slot 0); the rest run in pairs inside the recompute loop, each
        // recorded at the loop's slot, and an odd last step is host-launched.
        // The reversed steps then run in the reverse loop, slot k - 1 down
        // to 0.  Both loops are graphs of this call (they hold its buffers).
        rc = step_recorded(c, st, rec);
        if (rc) break;
        const uint32_t pairs = (k - 1) / 2;
        e = launch_set_words(c->loopCtl + kLoopRecReq, Words{{pairs, 0u, 1u, k, 0u, k - 1u}, 6u},
                             st);
        if (e != cudaSuccess) break;
        if (pairs) {
            const int p = c->cur;
            if (!recLoop[p]) {
                rc = build_while_graph(
                    c, kLoopRecReq, kLoopRecSlot, 2,
                    [&](cudaStream_t bs) {
                        return enqueue_step_pair(c, p, bs, [&](int k, cudaStream_t s2) {
                            return adj_record_step(
                                rec, RecSlot{c->loopCtl + kLoopRecSlot, (uint32_t)k, stepBytes},
                                c->n, c->numCells, step_in(c, p ^ k), step_in_static(c, p ^ k),
                                c->src, c->cells[p ^ k ^ 1], c->acc, c->alpha, s2);
                        });
                    },
                    &recLoop[p]);
                if (rc) break;
            }
            e = cudaGraphLaunch(recLoop[p], st);
            if (e != cudaSuccess) break;
        }
        if ((k - 1) & 1) {
            rc = step_recorded(c, st, rec + stepBytes * (k - 1));
            if (rc) break;
        }
        if (!revLoop) {
            rc = build_while_graph(
                c, kLoopRevReq, kLoopRevSlot, -1,
                [&](cudaStream_t bs) {
                    return adj_backward_step(c->P, c->nspec ? c->dTable : nullptr, c->spec, rec,
                                             RecSlot{c->loopCtl + kLoopRevSlot, 0u, stepBytes}, n,
                                             c->numCells, reinterpret_cast<float2*>(lamPos),
                                             reinterpret_cast<float2*>(lamVel), lamOmega, tlx,
                                             tlv, tlw, lamF, lamM, acc, bs);
                },
                &revLoop);
            if (rc) break;
        }
        e = cudaGraphLaunch(revLoop, st);
    }
    if (rc == DEM_OK && e == cudaSuccess) e = adj_sum_coef(acc, n, first, ns, sum, st);
    if (rc == DEM_OK && e == cudaSuccess)
        e = cudaMemcpyAsync(grad, sum, 8ull * DEM_ADJ_NUM_COEF * ns, cudaMemcpyDeviceToHost, st);
    // the buffers and loops stay for the next call: wait for this one's work
    // even when it failed part way
    const cudaError_t es = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = es;
    if (rc != DEM_OK || e != cudaSuccess) drop_adj_graphs(c);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "adjoint backward");
    return DEM_OK;
}
