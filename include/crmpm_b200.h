/*
 * crmpm_b200.h — C ABI of the B200-native MPM substep engine.
 *
 * This library replaces CRESSim-MPM's GPU solvers (src/solver/gpu_*_mpm_solver.cu) behind the
 * reference's own solver interface (include/solver/mpm_solver.h:63-191,
 * src/solver/mpm_solver_base.h:41-171, src/solver/mpm_solver_gpu.h:43-57).  Every entry point
 * below names the reference member it stands in for.  All pointers handed to a solver are DEVICE
 * pointers unless the argument name ends in "Host"; every call is asynchronous on the solver's
 * CUDA stream except where stated.
 *
 * Error convention: every function returns CRB200_OK (0) or a negative CRB200_ERR_* code and
 * records a message readable with CrB200GetLastError().  The reference logs CUDA errors and
 * continues (src/utils/check_cuda.cuh:35-44); this library reports them instead.
 *
 * The struct layouts below are field-for-field the layouts of the reference's SoA descriptors so
 * that a reference-side adapter can pass its own structs by reinterpretation:
 *   CrB200ShapeData       == crmpm::ShapeData        (include/engine/shape.h:58-89)
 *   CrB200GeometryData    == crmpm::GeometryData     (include/engine/geometry.h:65-108)
 *   CrB200GeometrySdfData == crmpm::GeometrySdfData  (include/engine/geometry.h:113-118)
 * Vec3f and Quat are 16-byte float4 in the reference (include/math/vec3.h:388-396,
 * include/math/quat.h:48-56); they appear here as CrB200Float4.
 */
#ifndef CRMPM_B200_H
#define CRMPM_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define CRB200_API __attribute__((visibility("default")))
#else
#define CRB200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------------------------ */
/* Status codes                                                                                */
/* ------------------------------------------------------------------------------------------ */

#define CRB200_OK 0
#define CRB200_ERR_INVALID_ARGUMENT (-1)
#define CRB200_ERR_NOT_INITIALIZED (-2)
#define CRB200_ERR_UNSUPPORTED (-3)
#define CRB200_ERR_CUDA (-4)
#define CRB200_ERR_OUT_OF_MEMORY (-5)
#define CRB200_ERR_CAPACITY (-6)
#define CRB200_ERR_TIMEOUT (-7)
#define CRB200_ERR_NUMERICS (-8)

/* Device status word bits, see CrB200SolverGetStatus(). */
#define CRB200_STATUS_NAN_STATE 0x1u      /* NaN/Inf found in particle position or velocity */
#define CRB200_STATUS_BLOCK_OVERFLOW 0x2u /* a grid block held more particles than a tile pass */
#define CRB200_STATUS_OUT_OF_DOMAIN 0x4u  /* a particle started a substep outside the grid     */

/* MpmSolverType values (include/solver/mpm_solver.h:51-61).  Only the GPU kinds are accepted:
 * the CPU kinds belong to the reference and have no counterpart here. */
#define CRB200_SOLVER_GPU_MLS 1
#define CRB200_SOLVER_GPU_PB 3
#define CRB200_SOLVER_GPU_STANDARD 5

/* ShapeContactModel (include/solver/mpm_solver.h:45-49). */
#define CRB200_CONTACT_KINEMATIC 0
#define CRB200_CONTACT_EFFECTIVE_MASS 1

/* ParticleMaterialType (include/solver/material_data.h:44-49). */
#define CRB200_MATERIAL_COROTATIONAL 0
#define CRB200_MATERIAL_NEOHOOKEAN 1
#define CRB200_MATERIAL_LINEAR_ELASTIC 2

/* ShapeType (include/engine/shape.h:47-52). */
#define CRB200_SHAPE_STATIC 0
#define CRB200_SHAPE_KINEMATIC 1
#define CRB200_SHAPE_DYNAMIC 2

/* GeometryType (include/engine/geometry.h:41-59). */
#define CRB200_GEOM_BOX 0
#define CRB200_GEOM_SPHERE 1
#define CRB200_GEOM_PLANE 2
#define CRB200_GEOM_CAPSULE 3
#define CRB200_GEOM_TRIANGLE_MESH 4
#define CRB200_GEOM_QUAD_SLICER 5
#define CRB200_GEOM_TRIANGLE_MESH_SLICER 6
#define CRB200_GEOM_CONNECTED_LINE_SEGMENTS 7
#define CRB200_GEOM_ARC 8

/* ------------------------------------------------------------------------------------------ */
/* Plain data descriptors                                                                      */
/* ------------------------------------------------------------------------------------------ */

typedef struct CrB200Float4 { float x, y, z, w; } CrB200Float4;
typedef struct CrB200Int4 { int x, y, z, w; } CrB200Int4;

/* Rigid shapes, struct-of-arrays, indexed by global shape id (include/engine/shape.h:58-89). */
typedef struct CrB200ShapeData {
    int *type;                     /* CRB200_SHAPE_* */
    int *geometryIdx;              /* geometry id of each shape */
    CrB200Float4 *position;        /* xyz */
    CrB200Float4 *rotation;        /* quaternion (x, y, z, w) */
    CrB200Float4 *invScale;        /* xyz */
    CrB200Float4 *linearVelocity;  /* xyz */
    CrB200Float4 *angularVelocity; /* xyz */
    CrB200Float4 *comInvMass;      /* centre of mass xyz, inverse mass w */
    CrB200Float4 *inertiaInv0;     /* inverse inertia, diagonal */
    CrB200Float4 *inertiaInv1;     /* inverse inertia, off-diagonal (xy, xz, yz) */
    CrB200Float4 *force;           /* output coupling force (dynamic shapes) */
    CrB200Float4 *torque;          /* output coupling torque (dynamic shapes) */
    CrB200Float4 *params0;         /* x smooth distance, y drag, z friction, w SDF fatten */
    int size;
} CrB200ShapeData;

/* Geometry, struct-of-arrays (include/engine/geometry.h:65-108). */
typedef struct CrB200GeometryData {
    int *type;             /* CRB200_GEOM_* */
    CrB200Float4 *params0; /* per-type parameters, integer fields bit-cast into floats */
    int size;
} CrB200GeometryData;

/* Precomputed SDF grids and line points (include/engine/geometry.h:113-118). */
typedef struct CrB200GeometrySdfData {
    CrB200Int4 *dimension;                /* per SDF id */
    CrB200Float4 *lowerBoundCellSize;     /* per SDF id: lower bound xyz, cell size w */
    CrB200Float4 *gradientSignedDistance; /* flattened grids: gradient xyz, distance w */
} CrB200GeometrySdfData;

typedef struct CrB200Solver *CrB200SolverHandle;

/* ------------------------------------------------------------------------------------------ */
/* Library                                                                                     */
/* ------------------------------------------------------------------------------------------ */

/* Message of the last failing call on this thread (empty string if none). */
CRB200_API const char *CrB200GetLastError(void);

/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
CRB200_API int CrB200GetVersion(void);

/* Number of CUDA kernels this library launched since load (all solvers, all threads). */
CRB200_API uint64_t CrB200GetKernelLaunchCount(void);

/* ------------------------------------------------------------------------------------------ */
/* Solver life cycle                                                                           */
/* ------------------------------------------------------------------------------------------ */

/* Create a solver.  Replaces the constructors GpuMlsMpmSolver(numParticles, cellSize, gridBound)
 * (src/solver/gpu_mls_mpm_solver.cu:40-52), GpuPbMpmSolver and GpuStandardMpmSolver, including
 * the node-count formula numNodesPerDim = int((max - min) / cellSize + 1) in float.
 * `stream` is a cudaStream_t (NULL = legacy default stream), as MpmSolverGpu::setCudaStream
 * (src/solver/mpm_solver_gpu.cpp:42-50). */
CRB200_API int CrB200SolverCreate(int solverType, int numMaxParticles, float cellSize,
                                  const float gridMin[3], const float gridMax[3], void *stream,
                                  CrB200SolverHandle *outSolver);

/* Free every device buffer the solver owns (MpmSolver release / GpuMlsMpmSolver::_release,
 * gpu_mls_mpm_solver.cu:111-124).  Bound buffers stay owned by the caller. */
CRB200_API int CrB200SolverRelease(CrB200SolverHandle solver);

/* MpmSolver::initialize (mpm_solver.h:70; gpu_mls_mpm_solver.cu:54-83): allocate solver-owned
 * state for numMaxParticles and zero it.  Particle data must be bound first. */
CRB200_API int CrB200SolverInitialize(CrB200SolverHandle solver);

/* MpmSolver::step (mpm_solver.h:75): one substep (PB-MPM: one step of `iterations` solver
 * iterations plus integration).  Writes the integration step size to *outDt (may be NULL). */
CRB200_API int CrB200SolverStep(CrB200SolverHandle solver, float *outDt);

/* Run `numSteps` steps back to back (the reference's `while (t < dt) t += step()` loop body
 * repeated, src/engine/scene_impl.cpp:313-317) without host round trips. */
CRB200_API int CrB200SolverStepMany(CrB200SolverHandle solver, int numSteps);

/* MpmSolver::fetchResults (mpm_solver_gpu.cpp:37-40): wait for the solver stream. */
CRB200_API int CrB200SolverFetchResults(CrB200SolverHandle solver);

/* MpmSolver::computeInitialData (mpm_solver.h:86-87; gpu_mls_mpm_solver.cu:85-100): F = I and
 * initial volume V0 = m / (sum_n w * m_n / dx^3) for the listed particles.  `indicesDevice` holds
 * `numParticles` particle indices in device memory. */
CRB200_API int CrB200SolverComputeInitialData(CrB200SolverHandle solver, unsigned int numParticles,
                                              const unsigned int *indicesDevice);

/* SceneImpl::_advanceTaskFn (src/engine/scene_impl.cpp:308-330): run substeps with the
 * reference's float accumulation `while (t < dt) t += step()`, then copy positionMass and
 * velocity of particles [0, numActive) into the host buffers (either may be NULL) as
 * SceneImpl::afterAdvance does (:249-263), and wait for the stream.  Host buffers should be
 * pinned for full copy bandwidth.  Writes the number of substeps taken to *outSubsteps. */
CRB200_API int CrB200SolverAdvance(CrB200SolverHandle solver, float dt, CrB200Float4 *positionMassHost,
                                   CrB200Float4 *velocityHost, int *outSubsteps);

/* Asynchronous CrB200SolverAdvance, as the reference's Scene::advance / fetchResults pair works
 * (scene_impl.cpp:290-330: advance starts the task, fetchResults waits): the substeps, a device
 * snapshot of positionMass and velocity and its copy into the host buffers (on a separate copy
 * stream) are enqueued and the call returns, so that the next call's substeps run while this
 * call's copy is in flight.  The host buffers must not be read or freed before
 * CrB200SolverFetchResults returns, which waits for the substeps and all copies; copies into one
 * buffer happen in call order, so a buffer may be passed again (alternating two buffer pairs lets
 * the caller read one frame while the next is copied).  Needs a non-default solver stream. */
CRB200_API int CrB200SolverAdvanceAsync(CrB200SolverHandle solver, float dt, CrB200Float4 *positionMassHost,
                                        CrB200Float4 *velocityHost, int *outSubsteps);

/* ------------------------------------------------------------------------------------------ */
/* Setters and binders (MpmSolver, mpm_solver.h:80-184; MpmSolverBase, mpm_solver_base.h)      */
/* ------------------------------------------------------------------------------------------ */

CRB200_API int CrB200SolverSetGravity(CrB200SolverHandle solver, float gx, float gy, float gz);
CRB200_API int CrB200SolverSetIntegrationStepSize(CrB200SolverHandle solver, float dt);
CRB200_API int CrB200SolverSetSolverIterations(CrB200SolverHandle solver, int iterations);
CRB200_API int CrB200SolverSetShapeContactModel(CrB200SolverHandle solver, int contactModel);
CRB200_API int CrB200SolverSetNumActiveParticles(CrB200SolverHandle solver, unsigned int n);

/* bindParticleData (mpm_solver.h:101): positionMass float4[numMaxParticles] (xyz position,
 * w mass) and velocity float4[numMaxParticles] (xyz).  Both device pointers, 16-byte aligned. */
CRB200_API int CrB200SolverBindParticleData(CrB200SolverHandle solver, CrB200Float4 *positionMass,
                                            CrB200Float4 *velocity);

/* bindParticleMaterials (mpm_solver.h:108): params0 float4 (x lambda, y mu for MLS/standard;
 * x elastic relaxation, y elasticity ratio for PB-MPM) and type int (CRB200_MATERIAL_*). */
CRB200_API int CrB200SolverBindParticleMaterials(CrB200SolverHandle solver, CrB200Float4 *params0,
                                                 int *type);

/* bindActiveMask (mpm_solver.h:125): uint8 per particle, nonzero = active. */
CRB200_API int CrB200SolverBindActiveMask(CrB200SolverHandle solver, unsigned char *activeMask);

CRB200_API int CrB200SolverSetNumShapes(CrB200SolverHandle solver, int numShapes);
CRB200_API int CrB200SolverBindShapeIds(CrB200SolverHandle solver, int *shapeIds);
CRB200_API int CrB200SolverBindShapeData(CrB200SolverHandle solver, const CrB200ShapeData *shapes);
CRB200_API int CrB200SolverBindGeometryData(CrB200SolverHandle solver,
                                            const CrB200GeometryData *geometries);
CRB200_API int CrB200SolverBindGeometrySdfData(CrB200SolverHandle solver,
                                               const CrB200GeometrySdfData *sdf);

/* ------------------------------------------------------------------------------------------ */
/* Introspection (no reference counterpart; the reference keeps F, C and V0 private)           */
/* ------------------------------------------------------------------------------------------ */

/* Grid node counts per dimension, as the reference computes them. */
CRB200_API int CrB200SolverGetGridDims(CrB200SolverHandle solver, int outDims[3]);

/* Copy solver-owned particle state for particles [0, n) to device buffers (any may be NULL):
 * F and C as float[n*9] column-major per particle (F(r,c) at 3*c + r), V0 as float[n]. */
CRB200_API int CrB200SolverCopyParticleState(CrB200SolverHandle solver, unsigned int n, float *F,
                                             float *C, float *V0);

/* Overwrite solver-owned particle state for particles [0, n) from device buffers (any may be
 * NULL; same layouts as CrB200SolverCopyParticleState). */
CRB200_API int CrB200SolverSetParticleState(CrB200SolverHandle solver, unsigned int n,
                                            const float *F, const float *C, const float *V0);

/* The engine's sort of the current positions (the binning of the reference's cell keys,
 * mls_mpm_algorithm.h:170-175): per-particle block key (uint32, key of an inactive particle is
 * 0xFFFFFFFF) and the canonical permutation (particle ids ordered by key, ties by id) of the
 * `*outNumSorted` binned particles.  Device buffers of numMaxParticles entries. */
CRB200_API int CrB200SolverCopySortState(CrB200SolverHandle solver, unsigned int *keys,
                                         unsigned int *sortedIds, unsigned int *outNumSortedHost);

/* Slicer cut masks of the most recent substep (bit i*9 + j*3 + k set when particle and stencil
 * node (i, j, k) lie on different sides of a slicer; mls_mpm_algorithm.h:200-210), evaluated on
 * the positions the substep started from.  Device buffer of numActive uint32; all zero when the
 * scene has no slicer shape. */
CRB200_API int CrB200SolverCopyCutMasks(CrB200SolverHandle solver, unsigned int *masks);

/* Sticky device status word (CRB200_STATUS_*), read with a bounded wait of timeoutMs
 * milliseconds on the solver stream; returns CRB200_ERR_TIMEOUT if the stream is still busy. */
CRB200_API int CrB200SolverGetStatus(CrB200SolverHandle solver, unsigned int *outStatusHost,
                                     int timeoutMs);
CRB200_API int CrB200SolverClearStatus(CrB200SolverHandle solver);

/* Option switches: CRB200_OPT_PHASE_TIMING records CUDA events around the phases of every
 * substep (see CrB200SolverGetPhaseTimes); it disables CUDA-graph replay while on.
 * CRB200_OPT_DETERMINISTIC_COUPLING makes the momentum that grid contact exchanges with dynamic
 * shapes (the force and torque accumulated into ShapeData, mpm_rigid_contact.h:59-82, 380-389)
 * independent of thread scheduling: per 4x4x4 grid block in a fixed order, then over blocks in
 * ascending order, instead of float atomics in arrival order.  Covers the first 4 dynamic shapes
 * of a scene (later ones keep the atomics); single-scene solvers only (CRB200_ERR_UNSUPPORTED on a
 * batch).  The first switch-on allocates 128 bytes per grid block. */
#define CRB200_OPT_PHASE_TIMING 3
#define CRB200_OPT_DETERMINISTIC_COUPLING 4
/* CRB200_OPT_DETERMINISTIC: substeps reproducible bit for bit from the same state.  On top of the
 * deterministic coupling, P2G adds nothing atomically: each 4x4x4 cell block stores its whole 6x6x6
 * node tile (3.4 KB per grid block, allocated at the first switch-on) and the grid update sums the
 * tiles covering a node in a fixed order (the reference sums with float atomics in arrival order,
 * math_helpers.h:309-328).  Particles whose stencil leaves the grid still go through atomics.
 * On a batch solver the particle state becomes reproducible the same way, while the coupling force
 * and torque of dynamic shapes keep their float atomics (the fixed-order coupling reduction is for
 * single scenes).  The substeps an adjoint backward pass replays follow the option, so a recording
 * made with it on is replayed bit for bit. */
#define CRB200_OPT_DETERMINISTIC 5
/* CRB200_OPT_RESIDENT (off by default; no counterpart in the reference, whose solvers keep the
 * particles in the caller's order): single-scene MLS-MPM solvers keep their own copy of the
 * particle state in slots grouped by 4x4x4 grid block and cell, and one fused kernel per substep
 * does the G2P of one substep and the P2G of the next.  Results are the same as with the option off
 * up to the order of float sums.  After every step / stepMany call the bound positionMass and
 * velocity buffers hold the state, as with the option off; edits to them between calls are read at
 * the next call.  A changed active mask or particle material takes effect at the next call after
 * BindActiveMask / BindParticleMaterials / SetNumActiveParticles / ComputeInitialData (the
 * reference's scene makes one of these whenever it changes them).  Deterministic substeps, adjoint
 * replays and batches use the particle-id-ordered path. */
#define CRB200_OPT_RESIDENT 6
/* CRB200_OPT_STANDARD_GPU_SEMANTICS (standard MPM; off by default): inactive particles as the
 * reference's GPU solver treats them.  That solver reads the active mask in P2G only, so particles
 * below the active count that the mask switches off still move with the grid in G2P, and its
 * computeInitialData initialises particles 0..n-1 whatever the index list
 * (gpu_standard_mpm_solver.cu:210-212, 280-282, 357-359).  Off, the engine follows the reference's
 * CPU solver, which honours both.  The drop-in adapter for eGpuStandardMpmSolver turns it on. */
#define CRB200_OPT_STANDARD_GPU_SEMANTICS 7
CRB200_API int CrB200SolverSetOption(CrB200SolverHandle solver, int option, int value);

/* Phase timing (CRB200_OPT_PHASE_TIMING on): CUDA-event milliseconds accumulated per phase on the
 * solver stream since the last reset, and the number of substeps they cover.  Phases:
 * 0 shape gather + binning + scan + scatter + cut masks + per-block cell sort, 1 P2G (particle
 * records + cell accumulation), 2 grid update, 3 G2P (PB-MPM: G2P plus the integration kernel).
 * On the resident path (CRB200_OPT_RESIDENT): 0 the call's start (shape gather, re-sort when due),
 * 1 the call's first P2G and the fused G2P -> P2G kernels, 2 grid updates, 3 the call's last G2P.
 * Synchronizes the solver stream. */
#define CRB200_NUM_PHASES 4
CRB200_API int CrB200SolverGetPhaseTimes(CrB200SolverHandle solver, float outMs[CRB200_NUM_PHASES],
                                         int *outSubsteps, int reset);

/* The fused G2P -> P2G kernel of the resident path (CRB200_OPT_RESIDENT) under phase timing:
 * CUDA-event milliseconds accumulated over its launches since the last reset, and their number
 * (no counterpart in the reference).  Synchronizes the solver stream. */
CRB200_API int CrB200SolverGetResidentKernelTime(CrB200SolverHandle solver, float *outMs, int *outLaunches,
                                                 int reset);

/* Launch-shape autotuner (no counterpart in the reference): times the candidate CTA counts of
 * the grid update (4, 8 or 16 per SM), the cell accumulation (1x or 2x its occupancy) and the
 * per-cell start computation (4 or 8 per SM) over substepsPerTrial substeps each (0: 8) from the current state, keeps the
 * fastest and restores the state; coupling forces of the trials are not reported.  Writes the
 * choice (update CTAs per SM, accumulation multiple, sort multiple) to outChoiceHost[3] if
 * given.  On the resident path (CRB200_OPT_RESIDENT) the second entry is the fused kernel's
 * multiple of its occupancy (1x or 2x) and the third is 1.  Needs a non-default solver stream;
 * synchronizes it. */
CRB200_API int CrB200SolverAutotune(CrB200SolverHandle solver, int substepsPerTrial, int *outChoiceHost);

/* Grid bookkeeping of the most recent substep: particles binned, active blocks, blocks updated,
 * and nodes that received mass (the touched-node count of the roofline byte model). */
CRB200_API int CrB200SolverGetGridStats(CrB200SolverHandle solver, unsigned int outStats[4]);

/* Number of PB-MPM material-constraint evaluations since the solver was made (or the counter was
 * last cleared) whose single-precision SVD was ill-conditioned and redone in double precision (a
 * tiny smallest singular value, or an inverted matrix whose two smallest singular values nearly
 * tie).  The reference's svd3 (include/math/svd3.h:1265-1276) has no such branch.  Synchronizes
 * the solver stream; clears the counter when `reset` is non-zero. */
CRB200_API int CrB200SolverGetFp64Fallbacks(CrB200SolverHandle solver, unsigned int *outCountHost, int reset);

/* The engine's 3x3 SVD on `n` matrices (device arrays, column-major, 9 floats each), as the
 * PB-MPM material constraint uses it (the reference's svd3 / svd<4>, include/math/svd3.h:74-1276):
 * the single-precision factors U, V (rotations, column-major) and singular values S (3 floats,
 * sign of the determinant on the last), the rotation the constraint blends toward (R, the
 * transpose of the polar rotation, column-major), and per matrix fp64Used = 1 where that rotation
 * came from the double-precision redo.  *fp64Count (device, may be null) is increased by the number
 * of redone matrices.  Enqueued on `stream` (a cudaStream_t). */
CRB200_API int CrB200SvdBatch(unsigned int n, const float *A, float *U, float *V, float *S, float *R,
                              unsigned int *fp64Used, unsigned int *fp64Count, void *stream);

/* ------------------------------------------------------------------------------------------ */
/* Batches of independent scenes (SimulationFactory::advanceAll, simulation_factory_impl.cpp:  */
/* 235-261 and 1106-1150, which loops over per-scene solvers; here all scenes advance in one   */
/* launch per phase)                                                                           */
/* ------------------------------------------------------------------------------------------ */

/* One scene of a batch: its grid, integration parameters, and its ranges in the shared particle
 * arrays and in the shared shape-id list.  Particle ranges of different scenes must not overlap. */
typedef struct CrB200BatchSceneDesc {
    float gridMin[3];
    float gridMax[3];
    float cellSize;
    float dt;
    float gravity[3];
    int contactModel;
    unsigned int particleOffset;
    unsigned int numParticles;
    int shapeOffset;
    int numShapes;
} CrB200BatchSceneDesc;

/* Create a solver that advances `numScenes` independent scenes together: every phase of a step
 * is one launch over all scenes (CrB200SolverStepMany replays it as one CUDA graph).  The returned
 * handle takes the ordinary solver calls: bind the shared particle, material, mask, shape-id,
 * shape, geometry and SDF arrays (ids in shape-id lists are global shape ids), Initialize,
 * ComputeInitialData (particle indices are global), Step / StepMany, CopyParticleState, Release.
 * All scenes share the solver type and PB-MPM iteration count; SetGravity /
 * SetIntegrationStepSize / SetShapeContactModel apply to every scene; the particle and shape
 * counts come from the descriptors (SetNumActiveParticles / SetNumShapes are refused). */
CRB200_API int CrB200BatchCreate(int solverType, int numScenes, const CrB200BatchSceneDesc *scenes,
                                 int numMaxParticles, int iterations, void *stream,
                                 CrB200SolverHandle *outSolver);

/* ------------------------------------------------------------------------------------------ */
/* Adjoint of the MLS-MPM substep (no counterpart in the reference: it has no gradient path)   */
/* ------------------------------------------------------------------------------------------ */

/* Run numSubsteps forward from the solver's current state and record the trajectory for
 * CrB200SolverAdjointBackward: the state (x, v, F, C) is kept every checkpointInterval substeps
 * (device memory, 104 bytes per particle per checkpoint) and the rest is recomputed backwards.
 * captureSubsteps (host, numCaptures entries, strictly increasing in [1, numSubsteps]) lists the
 * substeps whose positions are copied, as float4 (x, y, z, m), into capturedPositions (device,
 * numCaptures x numParticles entries, capture-major).  The solver is left in the final state.
 * Differentiated: the MLS-MPM solver, Neo-Hookean active particles, the kinematic and the
 * effective-mass contact models, box / sphere / plane / capsule shapes of uniform scale (anything
 * else, slicers included, is refused with CRB200_ERR_UNSUPPORTED).  Works on single-scene solvers
 * and batches alike. */
CRB200_API int CrB200SolverAdjointRecord(CrB200SolverHandle solver, int numSubsteps, int checkpointInterval,
                                         int numCaptures, const int *captureSubsteps,
                                         CrB200Float4 *capturedPositions);

/* Reverse pass over the recorded trajectory.  gradPositions (device, same layout as
 * capturedPositions; w ignored) holds dL/dx at each captured substep.  Outputs (device, one float4
 * per particle; any may be NULL): gradVelocity = dL/dv of the recorded initial state,
 * gradMaterial = (dL/dlambda, dL/dmu, 0, 0) summed over all substeps (lambda, mu = the
 * particle's params0.x / .y), gradPosition = dL/dx of the initial state with the rest volume V0
 * held fixed.  Gradients with respect to Young's modulus and Poisson's ratio follow by the chain
 * rule through lambda(E, nu), mu(E, nu).  Leaves the solver in the recorded final state. */
CRB200_API int CrB200SolverAdjointBackward(CrB200SolverHandle solver, const CrB200Float4 *gradPositions,
                                           CrB200Float4 *gradVelocity, CrB200Float4 *gradMaterial,
                                           CrB200Float4 *gradPosition);

/* ------------------------------------------------------------------------------------------ */
/* MLS-MPM substep without allocation (no counterpart in the reference)                        */
/* ------------------------------------------------------------------------------------------ */

/* Everything one allocation-free MLS-MPM substep reads and writes.  All pointers are device
 * pointers owned by the caller.  F and C are float[9 * numParticles], column-major per particle
 * (the layout of CrB200SolverCopyParticleState); they, positionMass and velocity are updated in
 * place.  Grid bounds, cell size, dt, gravity, shapes and contact model mean what they mean for a
 * solver created with CrB200SolverCreate. */
typedef struct CrB200NoAllocStep {
    float gridMin[3];
    float gridMax[3];
    float cellSize;
    float dt;
    float gravity[3];
    int contactModel;
    unsigned int numParticles;
    CrB200Float4 *positionMass;
    CrB200Float4 *velocity;
    float *F;
    float *C;
    const float *V0;
    const CrB200Float4 *matParams;
    const int *matType;
    const unsigned char *activeMask;
    int numShapes;
    const int *shapeIds;
    CrB200ShapeData shapes;
    CrB200GeometryData geometries;
    CrB200GeometrySdfData sdf;
} CrB200NoAllocStep;

/* One MLS-MPM substep that allocates no device or host memory, for callers that cannot call
 * cudaMalloc where they step the simulation (a host that pre-partitions all device memory, a
 * real-time loop that must not block on an allocation, code that only owns the buffers it was
 * handed).  This entry point has no counterpart in the reference.  Its grid scratch is a fixed
 * static device array of 2 x 262,144 nodes (8 MiB), held by every GPU that loads the library:
 * grids above 262,144 nodes (or more than 64 shapes) are rejected with CRB200_ERR_CAPACITY.  All
 * calls share that array, so calls that overlap on the GPU race; serialise them.  The first call on
 * a device looks up the array's address and should come before any stream capture; that address
 * is kept for the life of the process, so resetting the device afterwards is not supported.
 * positionMass, velocity, matParams and the shape / geometry float4 arrays must be 16-byte
 * aligned, and with shapes every shape array the substep reads (type, geometryIdx, position,
 * rotation, invScale, linearVelocity, angularVelocity, params0) and writes (force, torque) must be
 * non-null (CRB200_ERR_INVALID_ARGUMENT otherwise).  Every shapeIds entry must lie in
 * [0, shapes.size) and every geometryIdx in [0, geometries.size), as for the regular solver.  The
 * substep is enqueued on `stream` (a cudaStream_t, NULL = legacy default stream). */
CRB200_API int CrB200MlsSubstepNoAlloc(const CrB200NoAllocStep *step, void *stream);

/* ------------------------------------------------------------------------------------------ */
/* Triangle-mesh SDF grids built on the GPU (crmpm::SdfBuilder,                                */
/* include/geometry_utils/sdf_builder.h:46-98, src/geometry_utils/sdf_builder.cpp:84-368)     */
/* ------------------------------------------------------------------------------------------ */

/* crmpm::TriangleMesh (include/geometry_utils/triangle_mesh.h:39-46): HOST arrays, points as
 * numPoints x 3 floats, triangles as numTriangles x 3 vertex indices. */
typedef struct CrB200TriangleMesh {
    const float *points;
    const unsigned int *triangles;
    int numPoints;
    int numTriangles;
} CrB200TriangleMesh;

/* crmpm::SdfDesc (include/geometry_utils/sdf_builder.h:46-66).  The caller sets cellSize, fatten
 * and (slicer meshes only) slicerSpineArea, whose x is NaN when the slicer has no spine plane;
 * CrB200SdfPrecomputeDesc fills in the rest. */
typedef struct CrB200SdfDesc {
    float cellSize;
    float fatten;
    CrB200Float4 slicerSpineArea;
    float boundingSize[3];
    float lowerBound[3];
    int sdfDimension[3];
} CrB200SdfDesc;

/* SdfBuilder::precomputeSdfDesc (sdf_builder.cpp:84-103): the grid the reference lays over a mesh.
 * Its box is the union of the triangles' boxes, each enlarged by 1e-4 (winding_number.h:145-156),
 * then by `fatten`; like the reference's, each triangle box also contains the origin, because its
 * corners start at (0, 0, 0) before the vertices are included.  sdfDimension = int(size / cell + 1)
 * per axis.  Host only. */
CRB200_API int CrB200SdfPrecomputeDesc(CrB200SdfDesc *desc, const CrB200TriangleMesh *mesh);

/* SdfBuilder::computeSdf followed by computeSdfGradient (sdf_builder.cpp:105-161, 231-340), the
 * sequence of SimulationFactoryImpl::createGeometry for eTriangleMesh
 * (simulation_factory_impl.cpp:630-641).  Writes sdfDimension[0] x [1] x [2] float4 nodes (x
 * fastest) at gradientSignedDistance (DEVICE pointer): w = distance to the closest point on the
 * mesh, negative where the winding number of the mesh exceeds 0.5; xyz = its finite-difference
 * gradient, normalised when normalizeGradient is nonzero.  `desc` must come from
 * CrB200SdfPrecomputeDesc for the same mesh; every axis needs at least 2 nodes.  Enqueued on
 * `stream` (NULL = legacy default stream); the mesh arrays may be reused when the call returns. */
CRB200_API int CrB200SdfCompute(const CrB200SdfDesc *desc, const CrB200TriangleMesh *mesh,
                                CrB200Float4 *gradientSignedDistance, int normalizeGradient, void *stream);

/* The slicer variant: SdfBuilder::computeModSdf, computeSdfGradient (normalised) and
 * postProcessModSdfGradient (sdf_builder.cpp:163-229, 231-340, 342-367), the sequence of
 * createGeometry for eTriangleMeshSlicer (simulation_factory_impl.cpp:669-684).  w = unsigned
 * distance; a node whose closest point lies on a boundary edge or boundary vertex of the mesh (an
 * edge with fewer than two triangles) is off the mesh and gets NaN in all four components, unless
 * desc->slicerSpineArea (x not NaN) puts it on the positive side of the spine plane.  The spine
 * plane itself, which the reference stores one element before the grid, is the caller's to write. */
CRB200_API int CrB200SdfComputeMod(const CrB200SdfDesc *desc, const CrB200TriangleMesh *mesh,
                                   CrB200Float4 *gradientSignedDistance, void *stream);

/* GPU times in ms of the two kernels of the most recent CrB200SdfCompute / CrB200SdfComputeMod
 * call made on this host thread: outMs[0] the distance (and sign or off-mesh flag) kernel, outMs[1]
 * the gradient kernel; waits for them.  Host-side preparation and the mesh upload are not
 * included.  No counterpart in the reference. */
CRB200_API int CrB200SdfGetLastKernelTime(float outMs[2]);

#ifdef __cplusplus
}
#endif

#endif /* CRMPM_B200_H */
