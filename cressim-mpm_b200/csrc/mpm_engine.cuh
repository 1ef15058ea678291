// Host-side solver object of the B200 MPM engine.  One Solver stands in for one of the reference's
// GPU solvers (src/solver/gpu_{mls,pb,standard}_mpm_solver.cu) and honours the MpmSolver interface
// (include/solver/mpm_solver.h:63-191) through the C ABI in capi.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/crmpm_b200.h"
#include "mpm_device.cuh"

namespace crb200
{
    // Grid geometry of one scene.  Nodes are stored block-major: 4x4x4-node blocks of 64 float4
    // (1 KiB), block (bx, by, bz) at linear index bx + nb.x * (by + nb.y * bz).
    struct GridGeom
    {
        float3 gmin, gmax;
        float dx, invDx, cellVol;
        int3 n;  // node counts per dimension
        int3 nb; // blocks per dimension
        unsigned blockBase;
    };

    // Everything a kernel needs to know about one scene.  A solver holds one (the reference's
    // single-scene solvers) or many (the batch); particles of scene s occupy
    // [particleBegin, particleBegin + numActive) of the shared particle arrays and its shapes are
    // shapeTable[shapeBegin, shapeBegin + numShapes).
    struct StepParams
    {
        GridGeom g;
        float dt;
        float3 gravity;
        float cutoff;
        int contactModel;
        int solverType;
        unsigned numActive;
        int numShapes;
        unsigned particleBegin;
        int shapeBegin;
        int pad;
    };

    // Scene lookup handed to every kernel.  With one scene the kernels use their StepParams
    // argument and never touch these tables.
    struct SceneTable
    {
        const StepParams *params;            // numScenes entries
        const unsigned short *particleScene; // scene of each particle (0xFFFF: none)
        unsigned *flags;                     // SF_* shape flags per scene
        int numScenes;
        unsigned numParticles;               // particles covered by all scenes
    };

    // Device-side sort / bookkeeping header (one per solver).
    struct SortHeader
    {
        unsigned numActiveBlocks;
        unsigned numTouchedBlocks;
        // resident path: particles of the last P2G that left their block (cleared with
        // numTouchedBlocks and touchedNodes by one memset before every P2G)
        unsigned resMovers;
        unsigned touchedNodes;
        unsigned numSorted;
        unsigned status;
        unsigned fp64Fallbacks;
        unsigned shapeFlags;
        unsigned recordsValid;   // set by G2P when it binned the particles and wrote the next P2G records
        unsigned pbRecordsValid; // PB-MPM: set by the G2P of an iteration that wrote the next iteration's records
        unsigned sortSkip;       // the sort kernels of this call return at once (resident path, no re-sort due)
        unsigned resForce;       // host: re-sort at the next resident call
        unsigned resFromPlanes;  // host: that re-sort takes F, C, V0 from the particle-id planes
        unsigned resOutside;     // particles of this call whose stencil left their block's window
        unsigned matMixed;       // the resident particles' materials differ (else matUniform holds them)
        unsigned pad;
        float4 matUniform; // lambda, mu, type (int bits), 0
    };

    // Resident particle state of the fused single-scene MLS path: slot s holds one particle, slots
    // grouped by the 4x4x4 grid block (and within it by the cell) the particle sat in at the last
    // re-sort.
    struct ResState
    {
        float4 *x;          // position, mass
        float4 *v;          // velocity, kept only in scenes with slicers (G2P of a cut particle
                            // starts from it); elsewhere the caller's buffer holds it between calls
        float *V0;          // initial volume
        float *F, *C;       // 9 planes of `stride` floats, element (r, c) in plane 3c + r; C is
                            // current only after the last substep of a call (the fused kernel
                            // uses each substep's C at once, and the next G2P replaces it)
        const float4 *mat;  // lambda, mu, type (int bits), 0
        const unsigned *id; // particle id of each slot
        unsigned *cut;      // slicer cut mask of the position the last P2G used
        unsigned stride;
    };

    class Solver
    {
    public:
        Solver(int solverType, int numMaxParticles, float cellSize, const float gmin[3], const float gmax[3],
               cudaStream_t stream);
        // A batch of independent scenes sharing particle and shape arrays (CrB200BatchCreate).
        Solver(int solverType, int numMaxParticles, const CrB200BatchSceneDesc *scenes, int numScenes, int iterations,
               cudaStream_t stream);
        ~Solver();

        int initialize();
        int step();
        int stepMany(int n);
        int computeInitialData(unsigned n, const unsigned *indices);
        int fetchResults();
        int copySortState(unsigned *keysOut, unsigned *idsOut);
        int autotune(int trial, int choice[3]);
        int p2gBase = 0, sortBase = 0; // occupancy-derived CTA counts the autotuner multiplies
        int advance(float dt, float4 *hostX, float4 *hostV, int *outSubsteps);
        int advanceAsync(float dt, float4 *hostX, float4 *hostV, int *outSubsteps);
        cudaStream_t copyStream = nullptr; // host readback of advanceAsync
        cudaEvent_t stagedEvent = nullptr, copiedEvent = nullptr;
        float4 *stageX = nullptr, *stageV = nullptr;
        int collectPhaseTimes();

        // configuration (MpmSolver setters / binders)
        int solverType;
        int numMaxParticles;
        GridGeom geom;
        // batch: per-scene descriptors, grids and ranges (empty for a single-scene solver)
        std::vector<CrB200BatchSceneDesc> batch;
        std::vector<GridGeom> batchGeom;
        StepParams *dParams = nullptr;
        unsigned short *dParticleScene = nullptr;
        unsigned *dSceneFlags = nullptr;
        bool isBatch() const { return !batch.empty(); }
        int numScenes() const { return isBatch() ? (int)batch.size() : 1; }
        unsigned totalParticles() const;
        int totalShapes() const;
        cudaStream_t stream;
        float dt = 0.002f; // MpmSolverBase default (mpm_solver_base.h:146)
        float3 gravity = {0.f, 0.f, 0.f};
        int iterations = 10; // GpuPbMpmSolver default (gpu_pb_mpm_solver.cuh:53)
        int contactModel = 0;
        unsigned numActive = 0;
        float4 *positionMass = nullptr;
        float4 *velocity = nullptr;
        float4 *matParams = nullptr;
        int *matType = nullptr;
        unsigned char *activeMask = nullptr;
        int numShapes = 0;
        int *shapeIds = nullptr;
        CrB200ShapeData shapes{};
        CrB200GeometryData geometries{};
        CrB200GeometrySdfData sdf{};
        bool phaseTiming = false;
        cudaEvent_t phaseEv[5] = {};
        float phaseMs[4] = {0, 0, 0, 0};
        int phaseSteps = 0;
        int markPhase(int k); // record event k when phase timing is on

        bool initialized = false;
        unsigned configVersion = 0; // bumped by every setter so captured graphs are refreshed

        // solver-owned device state
        float *F = nullptr;  // 9 planes of numMaxParticles floats, F(r,c) in plane 3c + r
        float *Cm = nullptr; // APIC matrix, same layout
        // where G2P writes the updated state when not in place (the adjoint's replay: the next
        // tape slot); null in an ordinary substep
        float4 *outX = nullptr, *outV = nullptr;
        float *outF = nullptr, *outC = nullptr;
        struct StateView
        {
            float4 *x = nullptr, *v = nullptr;
            float *F = nullptr, *C = nullptr;
        };
        float *V0 = nullptr;
        float4 *gridA = nullptr; // accumulation grid (zero outside a substep)
        float4 *gridV = nullptr; // velocity grid
        float4 *gridF = nullptr; // node force (standard MPM)
        unsigned *keys = nullptr, *ranks = nullptr, *sortedIds = nullptr;
        unsigned *cellCount = nullptr; // particles per cell (binning), cleared by k_cellStarts
        unsigned *cellStart = nullptr; // absolute first sorted slot of each cell of the active blocks
        unsigned *blockCount = nullptr, *blockStart = nullptr;
        unsigned *activeList = nullptr, *touchedList = nullptr;
        unsigned *tileSums = nullptr;
        unsigned char *blockFlags = nullptr;
        unsigned long long *blockShapeMask = nullptr; // shapes that can reach each block's region (particles)

        unsigned *cutMasks = nullptr;
        float4 *records = nullptr;        // P2G records in sorted order, 4 float4 per particle
        SortHeader *header = nullptr;
        ShapeRec *shapeTable = nullptr;
        unsigned totalBlocks = 0;
        unsigned numTiles = 0;
        int p2gCtas = 0;
        int sortCtas = 0;
        int updCtas = 0;
        int strideCtas = 0;
        int cellCtas = 0;

        cudaGraphExec_t graph = nullptr;
        unsigned graphVersion = ~0u;
        int graphKernels = 0;
        // The substeps of a call but its last: their G2P leaves the velocity and C to the P2G record
        // it writes for the next substep (leanG2P is set while this graph is captured).
        cudaGraphExec_t graphLean = nullptr;
        bool leanG2P = false;
        // step(): the record invalidation and one substep
        cudaGraphExec_t graphSingle = nullptr;
        unsigned graphSingleVersion = ~0u;
        int graphSingleKernels = 0;

        StepParams params() const;
        SceneTable sceneTable() const;
        std::vector<StepParams> allParams() const;
        int uploadParams();
        int launchStep();   // enqueue one step's kernels
        template <bool Multi>
        int launchStepT(bool recompute);

        // adjoint of the MLS-MPM substep (CrB200SolverAdjointRecord / AdjointBackward)
        int adjointRecord(int numSubsteps, int interval, const int *captures, int numCaptures, float4 *capturedX);
        int adjointBackward(const float4 *gradX, float4 *gradV0, float4 *gradMat, float4 *gradX0);
        int runBackward(const float4 *gradX, unsigned n, unsigned pg, size_t sb, int T, int K, int c);
        int captureGraph(int which, int k, cudaGraphExec_t *out, int *kernels);
        int adjointGraphs(int K);
        void releaseAdjointGraphs();
        std::vector<cudaGraphExec_t> adjReplayG, adjReverseG, adjReplayLastG;
        // the adjoint's per-slot tape of a replayed substep: its P2G grid, grid velocities and sort
        struct TapeSlot
        {
            float4 *gridA, *gridV;
            unsigned *sortedIds, *cellStart, *blockStart, *activeList, *touchedList;
            SortHeader *hdr;
        };
        unsigned char *adjTape = nullptr;
        size_t adjTapeCap = 0;
        int tapeActive = -1; // slot the running forward substep writes its tape to (-1: none)
        size_t tapeSlotBytes() const;
        TapeSlot tapeSlot(int k) const;
        template <bool Multi>
        int adjointSubstepTape(int k, const unsigned char *state);
        int adjGraphKernels[3] = {0, 0, 0};
        unsigned adjGraphVersion = ~0u;
        unsigned char *adjGraphSeg = nullptr, *adjGraphTape = nullptr;
        int replayBody(int k, size_t sb, bool last);
        StateView slotState(int k, size_t sb) const;
        StateView bindState(const StateView &v);
        int reverseBody(int k, size_t sb);
        void releaseAdjoint();
        int adjointCheck();
        int saveState(unsigned char *dst);
        int invalidateRecords();
        int loadState(const unsigned char *src);

        // one saved state (x, v, F, C) in the layout of the live arrays
        size_t stateBytes() const { return (size_t)numMaxParticles * (2 * sizeof(float4) + 18 * sizeof(float)); }
        int adjSubsteps = 0, adjInterval = 0;
        std::vector<int> adjCaptures;
        bool adjRecorded = false;
        bool adjReplay = false;           // substeps replayed by the adjoint send coupling forces to scratch
        unsigned char *adjCkpt = nullptr; // checkpoint states (every adjInterval substeps and the last)
        unsigned char *adjSeg = nullptr;  // the states of one segment, recomputed backwards
        size_t adjCkptCap = 0, adjSegCap = 0;
        float4 *aX = nullptr, *aV = nullptr, *aMat = nullptr; // adjoint of x, v; d/d(lambda, mu)
        float *aF = nullptr, *aC = nullptr;                   // adjoint of F, C (planes of stride numMaxParticles)
        float4 *gridG = nullptr;                               // adjoint of the grid velocity / momentum and mass
        float4 *adjForce = nullptr, *adjTorque = nullptr;      // coupling output of recomputed substeps
        int sortParticles(const StepParams &p, bool ignoreMask);
        void gatherShapes(cudaStream_t s);
        bool detCoupling = false;            // CRB200_OPT_DETERMINISTIC_COUPLING
        float4 *detPartials = nullptr;       // per block and dynamic slot: force, torque partial sums
        unsigned *detMask = nullptr;         // bit per block: detPartials holds sums for it
        bool detP2G = false;                 // CRB200_OPT_DETERMINISTIC
        float4 *detTiles = nullptr, *detTilesF = nullptr; // per block: its P2G tile (deterministic P2G)
        unsigned long long *detFixedMass = nullptr;       // fixed-point initial node masses
        int setDeterministicCoupling(bool on);
        int setDeterministic(bool on);
        int detLevel(bool recomputing) const;
        cudaStream_t sideStream = nullptr; // shape gather / cut masks beside the sort chain
        cudaEvent_t forkEvent = nullptr, joinEvent = nullptr;

        // Resident path (single-scene MLS-MPM): particle state kept in cell order between substeps,
        // one fused kernel per substep for G2P of substep k and P2G of substep k + 1, a re-sort only
        // when particles have left their blocks (resident.cuh).
        bool residentOn = false;            // CRB200_OPT_RESIDENT
        // CRB200_OPT_STANDARD_GPU_SEMANTICS: standard MPM as the reference's GPU solver runs it
        // (G2P ignores the active mask, computeInitialData takes particles 0..n-1)
        bool stdGpuSemantics = false;
        unsigned char *onesMask = nullptr;  // numMaxParticles ones
        unsigned *iotaIds = nullptr;        // 0, 1, ..., numMaxParticles - 1
        bool resValid = false;              // the resident arrays hold the current particle state
        bool resPlanesStale = false;        // F and C in the particle-id planes are older than the resident ones
        ResState res{};
        float4 *resX2 = nullptr, *resMat2 = nullptr; // re-sort scratch
        float *resV02 = nullptr, *resF2 = nullptr, *resC2 = nullptr;
        unsigned *resId2 = nullptr, *resSlotOf = nullptr;
        unsigned *touchedFlag = nullptr;    // per grid block: already in this substep's touched list
        int resCtas = 0;                    // CTAs of the fused kernel: occupancy x SMs x resMult
        int resMult = 1;                    // autotuned
        cudaGraphExec_t resGraph[3] = {nullptr, nullptr, nullptr}; // call start, middle substep, last substep
        unsigned resGraphVersion = ~0u;
        int resGraphKernels[3] = {0, 0, 0};
        float fusedMs = 0.f;                // phase timing: the fused kernel alone
        int fusedLaunches = 0;
        bool scratchCoupling = false;       // autotune trials: coupling forces go to scratch
        bool residentUsable() const;
        int residentAlloc();
        int residentStep(int n);
        int setStdGpuSemantics(bool on);
        int residentPiece(int which);       // 0 call start, 1 middle substep, 2 last substep
        int residentSyncPlanes();           // F, C back to the particle-id planes
        int residentRetire();               // planes synced, resident state dropped
        int copyCutMasks(unsigned *out);
    };

    // Grid of one scene (node counts as the reference's solver constructors compute them).
    GridGeom makeGridGeom(float cellSize, const float gmin[3], const float gmax[3], unsigned blockBase);

    // the device SVD on a batch of matrices (CrB200SvdBatch)
    int svdBatch(unsigned n, const float *A, float *U, float *V, float *S, float *R, unsigned *fp64Used,
                 unsigned *fp64Count, cudaStream_t stream);

    // error plumbing shared by the C ABI
    void setLastError(const std::string &msg);
    int cudaFail(cudaError_t e, const char *what);
    void noteLaunches(uint64_t n);
    const char *lastError();
    uint64_t launchCount();
} // namespace crb200
