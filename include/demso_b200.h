/*
 * demso_b200 -- C ABI of the B200-native DEM step.
 *
 * Drop-in for the per-timestep pipeline of DemSo (blumberg/DemSo): the host
 * launch layer src/functions.cu / src/functions.cuh and the step loop of
 * src/main.cu (SimLooping, main.cu:396-507).  Every entry point takes plain
 * pointers and sizes, returns an int status (DEM_OK = 0) instead of the
 * reference's silent `void`, never exits the process, and takes the CUDA
 * stream to run on as `void*` (a cudaStream_t; NULL = legacy default stream,
 * the reference's only stream).
 *
 * Data layout is the reference's SoA layout (functions.cu:68-99):
 *   pos, vel, acc : float[2*n] (float2 per particle)
 *   theta, omega, alpha, pressure : float[n]
 *   id, loc, type : uint32[n]          (loc is indexed by id)
 *   hash, index   : uint32[n]
 *   cellStart, cellEnd : uint32[gridSize[0]*gridSize[1]]; empty cells have
 *                        cellStart = 0xFFFFFFFF (cellEnd of an empty cell is
 *                        left unspecified, as in the reference)
 * plus two per-particle arrays the reference keeps per type:
 *   radius, mass  : float[n]
 * The reference stores radius/mass/inertia/coefficients per particle *type*
 * in constant memory (main.cuh:39-54, particles_kernel.cuh:31-33, at most 10
 * types).  Here radius and mass are per particle, inertia is 2/5 m r^2
 * evaluated as main.cu:193 does, and the contact coefficients come from a
 * material table of up to DEM_MAX_MATERIALS entries indexed by `type`
 * (`type` may be NULL when there is one material).
 *
 * All device pointers must be device-accessible and 8-byte aligned for the
 * float2 arrays.  Functions named *_host take host pointers.
 */
#ifndef DEMSO_B200_H
#define DEMSO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DEM_ABI_VERSION 2

#define DEM_OK 0
#define DEM_ERR_INVALID_ARG 1 /* bad pointer, size, grid (not a power of two) */
#define DEM_ERR_CUDA 2        /* a CUDA call failed; see dem_last_error_string */
#define DEM_ERR_OOB 3         /* a particle position became NaN/Inf */
#define DEM_ERR_TIMEOUT 4     /* a bounded device-side wait gave up */
#define DEM_ERR_NO_MEMORY 5   /* device allocation failed */
#define DEM_ERR_CAPACITY 6    /* more particles/cells than the context holds */

#define DEM_MAX_MATERIALS 10  /* MAX_PARTICLES_TYPES (main.cuh:33) */

/* Per-material contact coefficients: the reference's ParticleProperties
 * (main.cuh:39-54) minus radius/mass/inertia/colour.  Pair values follow the
 * reference: stiffness and damping combine in series, a*b/(a+b) (0 if either
 * is 0; particles_kernel.cuh:36-41, :269-274), friction by the mean (:275). */
typedef struct DemMaterial {
    float normalStiffness;     /* <stiffness dir="normal"> */
    float shearStiffness;      /* <stiffness dir="shear"> */
    float normalDamping;       /* <damping>, a dashpot coefficient [N s/m] */
    float boundaryDamping;     /* <damping type="boundary">: wall velocity factor */
    float frictionCoefficient; /* <friction> */
    float attractCoefficient;  /* <attraction>; 0 disables attractSpheres */
} DemMaterial;

/* Scene-wide parameters: the reference's SystemProperties (main.cuh:108-122)
 * plus the material table. */
typedef struct DemSystem {
    uint32_t numParticles;
    float cubeDimension[2];      /* box size Lx, Ly */
    uint32_t gridSize[2];        /* cells per axis; powers of two (hash wraps with a mask) */
    float timeStep;
    float gravity[2];
    float boundaryNormalStiffness; /* carried for completeness; the reference's
                                      floor law does not use it (particles_kernel.cuh:423-427) */
    float boundaryShearStiffness;
    uint32_t numMaterials;       /* 1..DEM_MAX_MATERIALS */
    DemMaterial materials[DEM_MAX_MATERIALS];
} DemSystem;

/* ---------------------------------------------------------------------------
 * Library
 * ------------------------------------------------------------------------- */
int dem_abi_version(void);
/* Text of the last error on the calling host thread ("" if none). */
const char* dem_last_error_string(void);
/* Validates a DemSystem (powers of two, material count, positive sizes). */
int dem_validate_system(const DemSystem* sys);

/* ---------------------------------------------------------------------------
 * Per-stage entry points: one per host wrapper of the reference's step.
 * Caller owns every buffer; outputs match the reference's per stage.
 * ------------------------------------------------------------------------- */

/* Replaces calcHash (functions.cu:315-327 -> calcHashD, particles_kernel.cuh:133-151):
 * gridParticleHash[i] = cell of pos[i], gridParticleIndex[i] = i. */
int dem_calc_hash(const DemSystem* sys, const float* pos, uint32_t* gridParticleIndex,
                  uint32_t* gridParticleHash, uint32_t numParticles, void* stream);

/* Scratch bytes dem_sort_particles needs for n pairs of `keyBits`-bit keys. */
size_t dem_sort_scratch_bytes(uint32_t numParticles, uint32_t keyBits);

/* Replaces sortParticles (functions.cu:336-341, thrust::sort_by_key): stable
 * ascending sort of (hash, index) pairs in place.  Only the low `keyBits`
 * bits of the keys are examined (keys must be < 2^keyBits; 32 = any key).
 * `scratch` is device memory of dem_sort_scratch_bytes() bytes. */
int dem_sort_particles(uint32_t* gridParticleHash, uint32_t* gridParticleIndex,
                       uint32_t numParticles, uint32_t keyBits, void* scratch,
                       size_t scratchBytes, void* stream);

/* No counterpart in the reference: dem_sort_particles for callers that
 * cannot allocate device memory -- step loops that must not stall on the
 * device-wide synchronisation that cudaMalloc/cudaFree can cause, and host
 * programs whose own memory manager owns every device allocation and hands
 * out no scratch.  Same stable in-place sort and result as
 * dem_sort_particles, but the scratch is a fixed array inside the library
 * (about 2.6 MB, held on every GPU that loads the library until exit), so at
 * most 262,144 pairs per call; larger calls fail with DEM_ERR_CAPACITY.
 * Allocates nothing.  The first call on a device looks up that array's
 * device address and keeps it for the life of the process; make that first
 * call before any stream capture.  A device reset after it (cudaDeviceReset,
 * or a reset of the primary context by other code in the process) is not
 * supported: the kept address would be stale.  All calls
 * share the array: calls that overlap on the GPU race and must be ordered on
 * one stream or synchronised. */
int dem_sort_particles_static(uint32_t* gridParticleHash, uint32_t* gridParticleIndex,
                              uint32_t numParticles, uint32_t keyBits, void* stream);

/* Replaces reorderDataAndFindCellStart (functions.cu:347-393 ->
 * reorderDataAndFindCellStartD, particles_kernel.cuh:156-233): marks every
 * cell empty, records [cellStart, cellEnd) of each occupied cell, gathers the
 * state into sorted order and scatters sortedLoc[id] = sorted position.
 * sortedType/oldType may be NULL (single material). */
int dem_reorder_data_and_find_cell_start(
    const DemSystem* sys, uint32_t* cellStart, uint32_t* cellEnd,
    float* sortedPos, float* sortedVel, float* sortedTheta, float* sortedOmega,
    float* sortedRadius, float* sortedMass, uint32_t* sortedID, uint32_t* sortedLoc,
    uint32_t* sortedType, const uint32_t* gridParticleHash, const uint32_t* gridParticleIndex,
    const float* oldPos, const float* oldVel, const float* oldTheta, const float* oldOmega,
    const float* oldRadius, const float* oldMass, const uint32_t* oldID, const uint32_t* oldType,
    uint32_t numParticles, uint32_t numCells, void* stream);

/* Replaces collide (functions.cu:398-467 -> collideD, particles_kernel.cuh:459-549,
 * without the control particle): gather-only 3x3-cell contact forces.
 * newAcc = F/m, newAlpha = M/I, pressure = the reference's diagnostic
 * (pressure may be NULL to skip it).  No atomics: results are deterministic. */
int dem_collide(const DemSystem* sys, const float* sortedPos, const float* sortedVel,
                float* newAcc, const float* sortedOmega, float* newAlpha,
                const uint32_t* sortedType, const float* sortedRadius, const float* sortedMass,
                const uint32_t* cellStart, const uint32_t* cellEnd, uint32_t numParticles,
                uint32_t numCells, float* pressure, void* stream);

/* Replaces integrateSystem (functions.cu:529-551 -> integrateSystemD,
 * particles_kernel.cuh:580-627): symplectic Euler, theta wrap, wall clamps
 * and floor contact, in place.  pressure may be NULL. */
int dem_integrate_system(const DemSystem* sys, float* pos, float* vel, const float* acc,
                         float* theta, float* omega, const float* alpha, const uint32_t* type,
                         const float* radius, const float* mass, float* pressure,
                         uint32_t numParticles, void* stream);

/* ---------------------------------------------------------------------------
 * Context API: the whole step (SimLooping's inner loop, main.cu:396-507)
 * on library-owned device buffers: a sort phase (incremental stable sort,
 * cell ranges, positions and radii moved to sorted order) and one step
 * kernel (collide, integrate, next hash, gathering the other fields into
 * sorted order), both replayed as CUDA graphs.  A context's calls share its
 * device buffers and its loop counters: issue them on one stream, or
 * synchronise before a call on another stream.  Different contexts are
 * independent and may run on different streams and host threads.
 * ------------------------------------------------------------------------- */
typedef struct DemContext DemContext;

/* Flags for dem_create. */
#define DEM_CTX_PRESSURE 1u   /* maintain the pressure diagnostic (as the reference does) */
#define DEM_CTX_ACCEL 2u      /* also store acc/alpha of the last step (output rows) */
#define DEM_CTX_DIRECT 4u     /* launch each kernel directly instead of through CUDA graphs
                                 (one host read-back per step; for per-kernel profiling) */
#define DEM_CTX_AUTOTUNE 8u   /* choose the step kernel's launch shape on the first steps
                                 (dem_get_step_variant) */
#define DEM_CTX_CALLER_STATE 16u /* allocate no particle state: the caller's buffers
                                    are handed over by dem_adopt_state */
#define DEM_CTX_RESIDENT 32u  /* run each dem_step call as one launch that keeps the
                                 particles in shared memory: batches as bins of
                                 specimens, one per multiprocessor (see
                                 dem_batch_create); single scenes of up to 8,192 disks
                                 as one thread-block cluster (see dem_step) */

int dem_create(const DemSystem* sys, uint32_t capacity, uint32_t flags, DemContext** out);
/* A context over the cell rows [rowFirst, rowFirst + rowCount) of sys's grid
 * (rowCount a power of two, at most gridSize[1]; rowFirst < gridSize[1]):
 * what a slab of a row decomposition steps.  Cells, keys and the sort span
 * only those rows, so a window of a tall scene sorts and scans its own cells,
 * not the scene's.  Positions give the scene's rows bit for bit (same box,
 * grid and walls); a row r then has the cell row (r - rowFirst) mod rowCount,
 * so the particles of rows [rowFirst, rowFirst + rowCount) are stepped
 * exactly as by a context over the whole grid (their neighbour rows must be
 * within the window too), while a particle outside them shares cells with
 * distant rows and misses its true neighbours, as one beyond a slab's edge
 * does.
 * dem_row_slots takes the scene's rows.  The cluster form of DEM_CTX_RESIDENT
 * and the adjoint take whole grids only.  rowFirst 0 and rowCount gridSize[1]
 * is dem_create.  No reference counterpart. */
int dem_create_rows(const DemSystem* sys, uint32_t capacity, uint32_t flags, uint32_t rowFirst,
                    uint32_t rowCount, DemContext** out);
int dem_destroy(DemContext* ctx);
/* Runtime parameter change (gravity, dt, materials; grid size and particle
 * count fixed): the reference's set_gravity (functions.cu:663-668) generalised. */
int dem_set_system(DemContext* ctx, const DemSystem* sys);

/* State transfer in the reference layout, any order of particles; ids must
 * be a permutation of 0..n-1 (loc is indexed by id).  `host` != 0: the
 * pointers are host memory (pinned or pageable), else device memory.
 * type may be NULL.  Reads the largest radius back (synchronises `stream`)
 * and clears the error word; the next step sorts from scratch.  The step
 * graphs already captured stay valid when n and the largest radius are those
 * of the previous state, and are captured again otherwise. */
int dem_set_state(DemContext* ctx, uint32_t n, const float* pos, const float* vel,
                  const float* theta, const float* omega, const float* radius,
                  const float* mass, const uint32_t* id, const uint32_t* type, int host,
                  void* stream);
/* Batched form: `numSpecimens` independent scenes stepped together, each with
 * its own particle count (specs[s].numParticles), box, grid, gravity, time
 * step and materials.  The state is the concatenation of the specimens
 * (specimen 0 first); ids are one permutation of 0..N-1 over the whole
 * batch and loc is indexed by them.  Every other context call
 * (dem_set_state with all N particles, dem_step, dem_get_state, dem_check,
 * dem_get_followed, profiling) works on a batch; dem_set_system does not.
 * Cell keys carry a per-specimen offset, so the one stable sort of the batch
 * is each specimen's own stable sort and every specimen evolves bit for bit
 * as it would alone.  No counterpart in the reference (one scene per
 * process).
 *
 * With DEM_CTX_RESIDENT in `flags`, a dem_step call on the batch is one
 * persistent kernel launch: the specimens are packed into bins of at most
 * 8,192 particles, 8,192 cells and 64 specimens, and each thread block (one
 * per multiprocessor) takes bins from a queue and runs all the call's steps
 * of a bin inside its shared memory (positions, velocities, spins and radii;
 * the sort only on steps after a particle changed cell).  The trajectories
 * are those of the graph path bit for bit.  The first such call packs the
 * bins and allocates their scratch (about 64 B per particle of the largest
 * bin, per multiprocessor) and synchronises `stream`.  A batch with more
 * than one material, attraction, a control particle or a specimen too large
 * for one bin, and calls made while profiling, take the graph path instead.
 * After a resident call the next graph-path step sorts from scratch. */
int dem_batch_create(const DemSystem* specs, uint32_t numSpecimens, uint32_t flags,
                     DemContext** out);
/* Slots [*firstSlot, *firstSlot + *count) of the state hold specimen s (fixed
 * for the life of the batch). */
int dem_batch_specimen(DemContext* ctx, uint32_t specimen, uint32_t* firstSlot, uint32_t* count);
/* Replaces every specimen's parameters (box, gravity, time step, wall and
 * contact coefficients) of a batch; grid sizes, particle counts and the
 * material layout stay those of dem_batch_create.  The new table is copied
 * on `stream`, after the steps already queued there, so steps issued before
 * the call use the old parameters and steps issued after it the new ones.
 * The next dem_step sorts from scratch.  No reference counterpart. */
int dem_batch_set_systems(DemContext* ctx, const DemSystem* specs, uint32_t numSpecimens,
                          void* stream);

/* Copies out the current state in its current (cell-sorted) order, plus loc
 * (indexed by id) and, when requested at create time, pressure/acc/alpha of
 * the last step.  NULL outputs are skipped. */
int dem_get_state(DemContext* ctx, float* pos, float* vel, float* theta, float* omega,
                  float* radius, float* mass, uint32_t* id, uint32_t* type, uint32_t* loc,
                  float* pressure, float* acc, float* alpha, int host, void* stream);

/* One set of particle-state buffers in device memory, the reference's
 * ParticlesValues pos1/vel1/theta1/omega1/ID1/type1 (or the ...2 set),
 * with per-particle radius and mass.  `pos` and `radius` hold
 * n + DEM_STATE_PAD elements: the step reads whole groups of sorted
 * positions and radii past the last particle (the values there are never
 * used).  float2 arrays (pos, vel) 8-byte aligned, the others 4-byte. */
#define DEM_STATE_PAD 8u
typedef struct DemStateSet {
    float* pos;       /* 2 (n + DEM_STATE_PAD) floats, x and y interleaved */
    float* vel;       /* 2 n */
    float* theta;     /* n */
    float* omega;     /* n */
    float* radius;    /* n + DEM_STATE_PAD */
    float* mass;      /* n */
    uint32_t* id;     /* n */
    uint32_t* type;   /* n; ignored (may be NULL) with one material */
} DemStateSet;

/* The reference's "adopt caller buffers" form of the state: allocateVectors
 * (functions.cu:68-149) leaves the two ping-pong sets to the caller, and
 * its step loop (main.cu:395-430) alternates between them.  The context
 * keeps no copy: it steps in `first` and `second` (two distinct,
 * non-overlapping sets of device buffers that outlive the context or the
 * next dem_adopt_state) for as long as it holds them.  `first` holds the
 * initial state of n particles in the layout of dem_set_state; `second` is
 * scratch.  Which buffers hold the state after a step is given by
 * dem_state_view; dem_set_state and dem_get_state copy into and out of the
 * adopted buffers.  Reads the largest radius back (synchronises `stream`),
 * clears the error word, and captures the step graphs again when a buffer,
 * n or the largest radius changed.  A context created with
 * DEM_CTX_CALLER_STATE allocates no state of its own and takes its state
 * only this way. */
int dem_adopt_state(DemContext* ctx, uint32_t n, const DemStateSet* first,
                    const DemStateSet* second, void* stream);
/* Device pointers of the current state (n particles in cell-sorted order),
 * adopted buffers or the context's own: positions in the first set's pos,
 * the other fields in set *setIndex (0 first, 1 second; may be NULL).
 * Valid until the next step, dem_set_state or dem_adopt_state; reading them
 * on another stream needs the usual synchronisation.  type is NULL with one
 * material. */
int dem_state_view(DemContext* ctx, DemStateSet* out, int* setIndex);

/* Advances `nsteps` full steps (hash, sort, reorder, collide, integrate).
 * Once the context holds a previous order (after its first step) and is
 * neither tuning nor profiling nor created with DEM_CTX_DIRECT, a call of
 * two or more steps runs them in pairs inside ONE graph launch: a
 * device-side loop (a CUDA graph WHILE node, its pair count written to the
 * device by a one-thread kernel before the launch and counted down there)
 * whose body is two whole steps, one per buffer parity; an odd
 * last step is one more ordinary step.  The loop runs the same kernels on
 * the same buffers as single calls, so the bits are those of nsteps calls
 * of one step.
 * With DEM_CTX_AUTOTUNE the context's first 24 steps run the step kernel's
 * launch shapes in turn, each timed by CUDA events on `stream`; the step
 * that completes the 24th waits for `stream` once and keeps the shape with
 * the smallest median time.  Every shape computes the same bits, so the
 * trajectory does not depend on the choice.
 * A single scene created with DEM_CTX_RESIDENT, of at most 8,192 disks and
 * 8,192 cells, one material, no attraction and no control particle, steps
 * each call as ONE launch of a thread-block cluster of 8 blocks: every block
 * keeps the whole scene's positions, velocities, spins and radii in its
 * shared memory, steps an eighth of the disks and writes their new state
 * into every block's copy through distributed shared memory.  The bits are
 * the graph path's.  Its first call allocates the cluster's scratch (about
 * 270 B per disk); the next graph-path step sorts from scratch.  Other
 * scenes, calls while profiling, and GPUs that cannot hold such a cluster
 * take the graph path. */
int dem_step(DemContext* ctx, uint32_t nsteps, void* stream);

/* Launch shapes of the step kernel (threads per block x blocks per SM its
 * registers are capped for): 0 = 128 x 8 (the default), 1 = 64 x 16,
 * 2 = 256 x 4, 3 = 128 x 6. */
#define DEM_STEP_VARIANTS 4
typedef struct DemStepVariant {
    int32_t variant;       /* the shape in use */
    uint32_t threads;      /* its threads per block (128 while a control particle is set) */
    uint32_t blocksPerSm;  /* its register cap as resident blocks per SM */
    int32_t tuned;         /* 1 chosen by DEM_CTX_AUTOTUNE, 0 fixed, -1 still timing */
    float medianMs[DEM_STEP_VARIANTS]; /* the tuner's median step-kernel times (0 unless tuned) */
} DemStepVariant;
/* Fixes the launch shape (ends any tuning in progress). */
int dem_set_step_variant(DemContext* ctx, int32_t variant);
int dem_get_step_variant(DemContext* ctx, DemStepVariant* out);

/* Cell ranges of the last step's reorder, written to caller device buffers
 * of numCells words each in the reference's layout (either may be NULL). */
int dem_get_cells(DemContext* ctx, uint32_t* cellStart, uint32_t* cellEnd, void* stream);

/* Reads the context's device error word (synchronises `stream`): DEM_OK;
 * DEM_ERR_OOB when a position became NaN or infinite; DEM_ERR_TIMEOUT when a
 * bounded wait of the sort gave up (the state is then invalid, though every
 * access stayed in bounds, and every later step sorts from scratch until
 * dem_set_state).  dem_set_state clears the word. */
int dem_check(DemContext* ctx, void* stream);

/* Test hooks, no reference counterpart.  They inject failures on the host or
 * through bounded waits; none faults or hangs the GPU.
 *  - dem_debug_fail_allocation(k): the k-th device allocation the contexts
 *    make from now on fails as if the device had run out of memory (the
 *    call then returns DEM_ERR_NO_MEMORY); 0 turns it off.
 *  - dem_debug_live_allocations(): device allocations the contexts hold.
 *  - dem_debug_sort_hold(ctx, tile, spinLimit): in the context's full sort,
 *    tile `tile` of every pass never publishes its counts, so the tile after
 *    it waits until its bounded wait runs out after `spinLimit` iterations
 *    (0: the normal limit) and sets DEM_ERR_TIMEOUT; tile 0xFFFFFFFF holds
 *    none (normal use). */
int dem_debug_fail_allocation(int nth);
long long dem_debug_live_allocations(void);
int dem_debug_sort_hold(DemContext* ctx, uint32_t holdTile, uint32_t spinLimit);

/* The slots [*first, *first + *count) of the current state whose cell (the
 * sort key of the last step's sort, which ordered the state) lies in grid
 * rows [rowLo, rowHi): one contiguous range, since keys are numbered row by
 * row.  Rows are the scene's; a row window (dem_create_rows) takes rows
 * within its own block and the grid.  A slab decomposition cuts its bands and
 * own rows this way.  Needs
 * a step since the last dem_set_state / dem_adopt_state; single scenes only;
 * synchronises `stream`.  No reference counterpart. */
int dem_row_slots(DemContext* ctx, uint32_t rowLo, uint32_t rowHi, uint32_t* first,
                  uint32_t* count, void* stream);

/* Number of kernels one dem_step(ctx, 1, ...) launches (library kernels
 * only; the cellStart memset is not counted). */
int dem_kernels_per_step(DemContext* ctx);

/* Followed-particle rows, the reference's per-step output (writeOutputFile,
 * functions.cu:608-661): for each id in `ids` (host array), 12 words
 *   id, type (uint32 bits), x, y, vx, vy, ax, ay, theta, omega, alpha, pressure
 * are gathered on the device by loc[id] and copied to `rows` (host memory,
 * 12*count words) with one transfer; acc/alpha/pressure need the matching
 * DEM_CTX_* flags (zeros otherwise).  Synchronises `stream`. */
int dem_get_followed(DemContext* ctx, const uint32_t* ids, uint32_t count, float* rows,
                     void* stream);
/* dem_get_followed without the wait: the gather and the copy are enqueued on
 * `stream` and the call returns, so the next dem_step can be queued while the
 * rows travel.  `rows` (host memory, pinned for the copy to overlap, or device
 * memory) must stay valid until `stream` has passed the copy; the caller
 * waits for it (an event or a stream synchronisation) before reading them.
 * The context's staging buffer is reused in stream order, so successive calls
 * belong on one stream.  More than 64 ids still wait between batches.  No
 * counterpart in the reference, whose per-step output is synchronous. */
int dem_get_followed_async(DemContext* ctx, const uint32_t* ids, uint32_t count, float* rows,
                           void* stream);

/* `nsteps` steps as dem_step, with after each step the rows dem_get_followed
 * would give for `ids` (host array of `count` ids < n, read before the call
 * returns): rows (host or device memory) receives nsteps * count * 12 words,
 * step-major, the rows of step k at rows + 12 * count * k.  This is the
 * reference's stepping loop with writeOutputFile after every step
 * (main.cu:396-507, functions.cu:608-661) in one call: pairs of steps run in
 * the device-side loop, each step's rows gathered on the device into a ring
 * of up to 64 MB, which reaches `rows` by one copy per chunk of steps.  The
 * copies are queued on `stream`: with pinned or device memory the rows are
 * complete once `stream` has synchronised (pageable memory is written before
 * each copy returns).  Bit for bit the rows and state of nsteps calls of
 * dem_step(ctx, 1) each followed by dem_get_followed.  The device copy of
 * the ids and the ring grow to the largest call so far: a call that needs
 * more of either than every earlier call frees and allocates them again
 * (cudaFree/cudaMalloc, which can wait for the device) and captures the
 * step loop's graphs again; a call no larger than an earlier one allocates
 * nothing.  Callers whose id count varies can make one call with the largest
 * count first.  A context created with DEM_CTX_RESIDENT steps these calls on
 * the graph path (same bits). */
int dem_step_followed(DemContext* ctx, uint32_t nsteps, const uint32_t* ids, uint32_t count,
                      float* rows, void* stream);

/* Stage timing inside dem_step.  Each step is two graph launches on the
 * caller's stream: the sort phase (incremental sort, or the full radix sort
 * with cell ranges and gather) and the step kernel.  After
 * dem_profile_begin(ctx, maxSteps) the next dem_step calls (up to maxSteps
 * steps in total) record CUDA events around the two launches;
 * dem_profile_end synchronises and returns the summed milliseconds
 *   ms[0] = sort phase (sort, cell ranges, positions and radii moved into
 *           sorted order),
 *   ms[1] = 0 (the reorder is split between the two phases),
 *   ms[2] = collide + integrate + next hash, with the gather of the other
 *           fields into sorted order
 * and the number of steps profiled. */
#define DEM_NUM_STAGES 3
int dem_profile_begin(DemContext* ctx, uint32_t maxSteps);
int dem_profile_end(DemContext* ctx, float* ms, uint32_t* steps);

/* The control ("big") particle of the reference built with USE_BIG_PARTICLE
 * 1 (main.cuh:29): a kinematic disk of `material` that every particle meets
 * after its 3x3 neighbour cells (particles_kernel.cuh:520-541: contact, and
 * attraction where a material attracts).  The reaction on it -- the sums of
 * -f.x, -f.y and -m / r * radius over the particles -- is reduced on the
 * device as the reference reduces it (reduceVecD over blocks of
 * min(512, n), functions.cu:486-519, then the block sums in order), with no
 * per-step copy to the host.  After every step the particle moves as the
 * reference's host moves it (main.cu:511-514): pos += drift (float += double),
 * then y < wrapYBelow -> wrapYTo and x > wrapXAbove -> wrapXTo (NaN: no
 * wrap); the reference's values are drift (0, -0.005), wrapY (-1, 10.5),
 * wrapX (Lx + 0.5, -0.5), start (5, 9.5), vel 0.  The control particle
 * takes a single scene (not a batch); a single-material context needs
 * material 0.  Off by default; no reference counterpart as a function. */
typedef struct DemControl {
    float pos[2], vel[2];
    float theta, omega, radius;
    uint32_t material;
    double drift[2];
    double wrapYBelow, wrapYTo;
    double wrapXAbove, wrapXTo;
} DemControl;
/* Sets (or, with NULL, removes) the control particle.  The new state is
 * copied on `stream`, after the steps already queued there. */
int dem_set_control(DemContext* ctx, const DemControl* control, void* stream);
/* Its current state and the reaction (fx, fy, moment) of the last step;
 * synchronises `stream`.  Either output may be NULL. */
int dem_get_control(DemContext* ctx, DemControl* control, float* reaction, void* stream);

/* ---------------------------------------------------------------------------
 * Headless output
 * ------------------------------------------------------------------------- */

/* Disk splat of the particles (plotParticles, functions.cu:557-599 ->
 * plotSpheresD, particles_kernel.cuh:629-718) into a device buffer of
 * imageDIMx * imageDIMy uchar4 pixels (RGBA, row y = 0 at the bottom of the
 * box), instead of the reference's GL pixel buffer.  Pixels, shading and
 * colours follow the reference; where its threads race (overlapping disks,
 * orientation lines over other disks) the result is deterministic: the
 * particle with the highest index colours a shared pixel and lines are drawn
 * after all disks. */
typedef struct DemRenderParams {
    uint32_t imageDIMx, imageDIMy;
    uint32_t bgColor;          /* every byte of the background (cudaMemset value) */
    uint32_t viewRotations;    /* draw each particle's orientation line */
    uint32_t colorByPressure;  /* colour by pressure / maxPressure on the reference's colour bar */
    float maxPressure;
    float color[DEM_MAX_MATERIALS][3];  /* per material, 0..255 */
} DemRenderParams;
/* Per-stage form: caller buffers; `owner` is device scratch of
 * imageDIMx * imageDIMy words; type and pressure may be NULL. */
int dem_render_particles(const DemSystem* sys, const float* pos, const float* theta,
                         const uint32_t* type, const float* radius, const float* pressure,
                         uint32_t numParticles, const DemRenderParams* params, uint32_t* owner,
                         void* image, void* stream);
/* The context's current state; the owner scratch is held by the context
 * (allocated on the first call, or when the image grows). */
int dem_render(DemContext* ctx, const DemRenderParams* params, void* image, void* stream);

/* ---------------------------------------------------------------------------
 * Adjoint (no counterpart in the reference): reverse-mode gradients of a
 * scalar loss of the final state with respect to the initial state and the
 * contact coefficients, for a context (a scene or a batch) of one material
 * per specimen, without attraction, created with DEM_CTX_ACCEL and with at
 * least 3 cells per axis.
 *
 * dem_adj_forward runs nsteps steps exactly as dem_step and keeps the state
 * every `every` steps (device memory held by the context).  The caller then
 * reads the final state, forms the loss cotangents and calls
 * dem_adj_backward, which re-runs each window from its checkpoint while
 * recording it and reverses its steps.  The branch taken by every contact,
 * wall and floor contact in the forward is kept in the reverse ("frozen"
 * contact set).  lamPos/lamVel/lamOmega are device arrays in particle-id
 * order: on entry the cotangents of the final pos (2n), vel (2n) and omega
 * (n), on return those of the initial state.  grad (host, DEM_ADJ_NUM_COEF
 * doubles per specimen; one specimen for a single scene) receives, for each
 * specimen, dL/d of its: pair normal stiffness, pair shear stiffness,
 * pair dashpot, pair friction (the series/mean values of
 * particles_kernel.cuh:269-275), then the floor's dashpot (the material's
 * normalDamping), friction and series shear stiffness
 * (particles_kernel.cuh:419-421).  Coefficient sums are in double, in a
 * fixed order (deterministic).  After
 * dem_adj_backward the context holds the state at the end of the first
 * window; set the state again before stepping on.  The backward restores
 * the checkpoints as they are: a dem_set_state between the two calls that
 * changes the particle count or the largest radius makes dem_adj_backward
 * fail with DEM_ERR_INVALID_ARG.  Each window's re-run and reversed steps
 * run as two device-side loops (graph WHILE nodes), so the host does not
 * wait between windows.
 * ------------------------------------------------------------------------- */
#define DEM_ADJ_NUM_COEF 7
int dem_adj_forward(DemContext* ctx, uint32_t nsteps, uint32_t every, void* stream);
int dem_adj_backward(DemContext* ctx, float* lamPos, float* lamVel, float* lamOmega,
                     double* grad, void* stream);

/* ---------------------------------------------------------------------------
 * Scene generation (host only, no GPU needed)
 * ------------------------------------------------------------------------- */

/* .dsml scenes: the reference's input format (DEMParser, parser.cpp:49-377;
 * DEMSimulation::loadFromFile, DEMSimulation.cpp:45-60) and its scene
 * construction (PrepareSim, main.cu:54-369, with createRectanglesD and
 * createTrianglesD, particles_kernel.cuh:43-111).  Particles are numbered
 * single particles first, then rectangles, then triangles; every particle
 * carries its type's radius and mass; the materials are the particle types in
 * file order.  Rectangle lattice points are jittered by (N(0,1) - 0.5) / 100
 * of the spacing from a generator seeded by `seed` (the reference seeds
 * cuRAND with time(NULL)); DEM_DSML_NO_JITTER uses a zero deviate.  Errors
 * (DEM_ERR_INVALID_ARG) carry the reference's parse messages.  The step has
 * no control particle (the reference built with USE_BIG_PARTICLE 0): a
 * <controlled> tag is reported (its type) but creates nothing. */
#define DEM_DSML_NO_JITTER 1u
typedef struct DemDsml DemDsml;
typedef struct DemDsmlInfo {
    uint32_t numParticles, numTypes, numFollowed, imageHeight;
    uint32_t numRectangles, numTriangles, numSingles;
    int32_t controlledType;  /* -1 without a <controlled> tag */
    float timeStep;          /* <timestep> */
    float simDuration;       /* <simduration> in seconds; -1 = run forever */
} DemDsmlInfo;
typedef struct DemDsmlType {
    char id[64], name[128];
    float mass, radius;
    float color[3];          /* 0..255 from color="rrggbb" (white by default) */
} DemDsmlType;
int dem_dsml_load(const char* path, uint64_t seed, uint32_t flags, DemDsml** out);
int dem_dsml_parse(const char* text, size_t length, uint64_t seed, uint32_t flags, DemDsml** out);
void dem_dsml_free(DemDsml* scene);
int dem_dsml_info(const DemDsml* scene, DemDsmlInfo* info);
/* The scene's DemSystem, with the reference's grid rule (main.cu:218-236). */
int dem_dsml_system(const DemDsml* scene, DemSystem* sys);
/* The initial state into host arrays of numParticles entries (pos and vel:
 * two per particle); NULL outputs are skipped. */
int dem_dsml_state(const DemDsml* scene, float* pos, float* vel, float* theta, float* omega,
                   float* radius, float* mass, uint32_t* id, uint32_t* type);
/* The followed particle ids (numFollowed entries): single particles marked
 * follow="true", then the <follow> entries of <parameters>. */
int dem_dsml_followed(const DemDsml* scene, uint32_t* ids);
int dem_dsml_type(const DemDsml* scene, uint32_t type, DemDsmlType* out);

/* Seeded random sequential placement of n non-overlapping disks of the given
 * radii in [0,Lx]x[0,Ly] (host arrays; pos receives 2n floats in the order of
 * `radius`).  Replaces the reference's wall-clock-seeded block generators
 * (createRectanglesD, particles_kernel.cuh:43-74; seed time(NULL), main.cu:291)
 * for scenes that must be reproducible.  Disks are placed largest first into
 * `strips` horizontal strips filled in parallel; each disk gets up to
 * `trials` uniform random trials, then a search over jittered lattice points
 * of random cells.  The result depends only on the arguments.  Returns
 * DEM_ERR_CAPACITY (with *placed < n, unplaced positions NaN) when the box
 * is too full. */
int dem_scene_rsa(uint32_t n, const float* radius, float Lx, float Ly, uint64_t seed,
                  uint32_t strips, uint32_t trials, float* pos, uint32_t* placed);

#ifdef __cplusplus
}
#endif
#endif /* DEMSO_B200_H */
