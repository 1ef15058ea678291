// extern "C" entry points of libcrmpm_b200.so (declared in include/crmpm_b200.h).  Each one stands
// in for the reference member named in the header; they only validate arguments and forward to
// the Solver object.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <new>
#include <thread>
#include <utility>
#include <vector>

#include "mpm_engine.cuh"

using crb200::Solver;

struct CrB200Solver
{
    Solver *s;
};

namespace
{
    int bad(const char *msg)
    {
        crb200::setLastError(msg);
        return CRB200_ERR_INVALID_ARGUMENT;
    }
    Solver *get(CrB200SolverHandle h) { return h ? h->s : nullptr; }
} // namespace

#define SOLVER_OR_FAIL(h)                          \
    Solver *s = get(h);                            \
    if (!s)                                        \
        return bad("null solver handle");

extern "C"
{
    CRB200_API const char *CrB200GetLastError(void) { return crb200::lastError(); }

    CRB200_API int CrB200GetVersion(void) { return 100; }

    CRB200_API uint64_t CrB200GetKernelLaunchCount(void) { return crb200::launchCount(); }

    CRB200_API int CrB200SolverCreate(int solverType, int numMaxParticles, float cellSize, const float gridMin[3],
                                      const float gridMax[3], void *stream, CrB200SolverHandle *outSolver)
    {
        if (!outSolver || !gridMin || !gridMax)
            return bad("CrB200SolverCreate: null argument");
        *outSolver = nullptr;
        if (solverType != CRB200_SOLVER_GPU_MLS && solverType != CRB200_SOLVER_GPU_PB &&
            solverType != CRB200_SOLVER_GPU_STANDARD)
        {
            crb200::setLastError("CrB200SolverCreate: only the GPU solver types (1, 3, 5) are provided");
            return CRB200_ERR_UNSUPPORTED;
        }
        if (numMaxParticles <= 0 || !(cellSize > 0.f))
            return bad("CrB200SolverCreate: numMaxParticles and cellSize must be positive");
        for (int d = 0; d < 3; ++d)
            if (!(gridMax[d] > gridMin[d]))
                return bad("CrB200SolverCreate: empty grid bounds");
        Solver *s = new (std::nothrow) Solver(solverType, numMaxParticles, cellSize, gridMin, gridMax,
                                              static_cast<cudaStream_t>(stream));
        if (!s)
            return bad("CrB200SolverCreate: out of host memory");
        if (s->geom.n.x < 5 || s->geom.n.y < 5 || s->geom.n.z < 5)
        {
            delete s;
            return bad("CrB200SolverCreate: the grid needs at least 5 nodes per dimension");
        }
        if ((double)s->totalBlocks * 64.0 >= 4294967295.0)
        {
            delete s;
            crb200::setLastError("CrB200SolverCreate: grid exceeds 2^32 nodes");
            return CRB200_ERR_CAPACITY;
        }
        CrB200Solver *h = new (std::nothrow) CrB200Solver{s};
        *outSolver = h;
        return CRB200_OK;
    }

    CRB200_API int CrB200BatchCreate(int solverType, int numScenes, const CrB200BatchSceneDesc *scenes,
                                     int numMaxParticles, int iterations, void *stream, CrB200SolverHandle *outSolver)
    {
        if (!outSolver || !scenes)
            return bad("CrB200BatchCreate: null argument");
        *outSolver = nullptr;
        if (solverType != CRB200_SOLVER_GPU_MLS && solverType != CRB200_SOLVER_GPU_PB &&
            solverType != CRB200_SOLVER_GPU_STANDARD)
        {
            crb200::setLastError("CrB200BatchCreate: only the GPU solver types (1, 3, 5) are provided");
            return CRB200_ERR_UNSUPPORTED;
        }
        if (numScenes <= 0 || numScenes > 65535)
            return bad("CrB200BatchCreate: numScenes must be in [1, 65535]");
        if (numMaxParticles <= 0 || iterations < 0)
            return bad("CrB200BatchCreate: numMaxParticles must be positive and iterations non-negative");
        // particle ranges: inside the arrays and pairwise disjoint
        std::vector<std::pair<unsigned, unsigned>> ranges;
        double nodes = 0.0;
        for (int i = 0; i < numScenes; ++i)
        {
            const CrB200BatchSceneDesc &d = scenes[i];
            if (!(d.cellSize > 0.f) || !(d.dt > 0.f))
                return bad("CrB200BatchCreate: cellSize and dt must be positive");
            for (int a = 0; a < 3; ++a)
                if (!(d.gridMax[a] > d.gridMin[a]))
                    return bad("CrB200BatchCreate: empty grid bounds");
            if (d.contactModel != CRB200_CONTACT_KINEMATIC && d.contactModel != CRB200_CONTACT_EFFECTIVE_MASS)
                return bad("CrB200BatchCreate: unknown contact model");
            if ((unsigned long long)d.particleOffset + d.numParticles > (unsigned long long)numMaxParticles)
            {
                crb200::setLastError("CrB200BatchCreate: a particle range exceeds numMaxParticles");
                return CRB200_ERR_CAPACITY;
            }
            if (d.numShapes < 0 || d.shapeOffset < 0)
                return bad("CrB200BatchCreate: negative shape range");
            if (d.numShapes > crb200::kMaxShapes)
            {
                crb200::setLastError("CrB200BatchCreate: at most 64 shapes per scene");
                return CRB200_ERR_CAPACITY;
            }
            if (d.numParticles)
                ranges.emplace_back(d.particleOffset, d.particleOffset + d.numParticles);
            const crb200::GridGeom g = crb200::makeGridGeom(d.cellSize, d.gridMin, d.gridMax, 0);
            if (g.n.x < 5 || g.n.y < 5 || g.n.z < 5)
                return bad("CrB200BatchCreate: every grid needs at least 5 nodes per dimension");
            nodes += 64.0 * g.nb.x * g.nb.y * (double)g.nb.z;
        }
        std::sort(ranges.begin(), ranges.end());
        for (size_t i = 1; i < ranges.size(); ++i)
            if (ranges[i].first < ranges[i - 1].second)
                return bad("CrB200BatchCreate: particle ranges of two scenes overlap");
        if (nodes >= 4294967295.0)
        {
            crb200::setLastError("CrB200BatchCreate: the scenes' grids exceed 2^32 nodes together");
            return CRB200_ERR_CAPACITY;
        }
        Solver *s = new (std::nothrow)
            Solver(solverType, numMaxParticles, scenes, numScenes, iterations, static_cast<cudaStream_t>(stream));
        if (!s)
            return bad("CrB200BatchCreate: out of host memory");
        CrB200Solver *h = new (std::nothrow) CrB200Solver{s};
        *outSolver = h;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverRelease(CrB200SolverHandle solver)
    {
        SOLVER_OR_FAIL(solver);
        delete s;
        delete solver;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverInitialize(CrB200SolverHandle solver)
    {
        SOLVER_OR_FAIL(solver);
        if (s->initialized)
            return bad("CrB200SolverInitialize: already initialized");
        return s->initialize();
    }

    CRB200_API int CrB200SolverStep(CrB200SolverHandle solver, float *outDt)
    {
        SOLVER_OR_FAIL(solver);
        int r = s->step();
        if (outDt)
            *outDt = s->dt;
        return r;
    }

    CRB200_API int CrB200SolverStepMany(CrB200SolverHandle solver, int numSteps)
    {
        SOLVER_OR_FAIL(solver);
        return s->stepMany(numSteps);
    }

    CRB200_API int CrB200SolverFetchResults(CrB200SolverHandle solver)
    {
        SOLVER_OR_FAIL(solver);
        return s->fetchResults();
    }

    CRB200_API int CrB200SolverComputeInitialData(CrB200SolverHandle solver, unsigned int numParticles,
                                                  const unsigned int *indicesDevice)
    {
        SOLVER_OR_FAIL(solver);
        return s->computeInitialData(numParticles, indicesDevice);
    }

    CRB200_API int CrB200SolverSetGravity(CrB200SolverHandle solver, float gx, float gy, float gz)
    {
        SOLVER_OR_FAIL(solver);
        s->gravity = make_float3(gx, gy, gz);
        for (auto &d : s->batch)
        {
            d.gravity[0] = gx;
            d.gravity[1] = gy;
            d.gravity[2] = gz;
        }
        s->configVersion++;
        return s->uploadParams();
    }

    CRB200_API int CrB200SolverSetIntegrationStepSize(CrB200SolverHandle solver, float dt)
    {
        SOLVER_OR_FAIL(solver);
        if (!(dt > 0.f))
            return bad("CrB200SolverSetIntegrationStepSize: dt must be positive");
        s->dt = dt;
        for (auto &d : s->batch)
            d.dt = dt;
        s->configVersion++;
        return s->uploadParams();
    }

    CRB200_API int CrB200SolverSetSolverIterations(CrB200SolverHandle solver, int iterations)
    {
        SOLVER_OR_FAIL(solver);
        if (iterations < 0)
            return bad("CrB200SolverSetSolverIterations: negative iteration count");
        s->iterations = iterations;
        s->configVersion++;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverSetShapeContactModel(CrB200SolverHandle solver, int contactModel)
    {
        SOLVER_OR_FAIL(solver);
        if (contactModel != CRB200_CONTACT_KINEMATIC && contactModel != CRB200_CONTACT_EFFECTIVE_MASS)
            return bad("CrB200SolverSetShapeContactModel: unknown contact model");
        s->contactModel = contactModel;
        for (auto &d : s->batch)
            d.contactModel = contactModel;
        s->configVersion++;
        return s->uploadParams();
    }

    CRB200_API int CrB200SolverSetNumActiveParticles(CrB200SolverHandle solver, unsigned int n)
    {
        SOLVER_OR_FAIL(solver);
        if (s->isBatch())
        {
            crb200::setLastError("CrB200SolverSetNumActiveParticles: a batch takes its particle ranges from its scenes");
            return CRB200_ERR_UNSUPPORTED;
        }
        if (n > (unsigned)s->numMaxParticles)
        {
            crb200::setLastError("CrB200SolverSetNumActiveParticles: more than numMaxParticles");
            return CRB200_ERR_CAPACITY;
        }
        if (int rc = s->residentRetire()) // the particle set changes: re-sort at the next resident call
            return rc;
        s->numActive = n;
        s->configVersion++;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverBindParticleData(CrB200SolverHandle solver, CrB200Float4 *positionMass,
                                                CrB200Float4 *velocity)
    {
        SOLVER_OR_FAIL(solver);
        if (!positionMass || !velocity)
            return bad("CrB200SolverBindParticleData: null pointer");
        if ((reinterpret_cast<uintptr_t>(positionMass) | reinterpret_cast<uintptr_t>(velocity)) & 15u)
            return bad("CrB200SolverBindParticleData: buffers must be 16-byte aligned");
        if (int rc = s->residentRetire())
            return rc;
        s->positionMass = reinterpret_cast<float4 *>(positionMass);
        s->velocity = reinterpret_cast<float4 *>(velocity);
        s->configVersion++;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverBindParticleMaterials(CrB200SolverHandle solver, CrB200Float4 *params0, int *type)
    {
        SOLVER_OR_FAIL(solver);
        if (!params0 || !type)
            return bad("CrB200SolverBindParticleMaterials: null pointer");
        if (int rc = s->residentRetire())
            return rc;
        s->matParams = reinterpret_cast<float4 *>(params0);
        s->matType = type;
        s->configVersion++;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverBindActiveMask(CrB200SolverHandle solver, unsigned char *activeMask)
    {
        SOLVER_OR_FAIL(solver);
        if (!activeMask)
            return bad("CrB200SolverBindActiveMask: null pointer");
        if (int rc = s->residentRetire())
            return rc;
        s->activeMask = activeMask;
        s->configVersion++;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverSetNumShapes(CrB200SolverHandle solver, int numShapes)
    {
        SOLVER_OR_FAIL(solver);
        if (s->isBatch())
        {
            crb200::setLastError("CrB200SolverSetNumShapes: a batch takes its shape ranges from its scenes");
            return CRB200_ERR_UNSUPPORTED;
        }
        if (numShapes < 0)
            return bad("CrB200SolverSetNumShapes: negative");
        if (numShapes > crb200::kMaxShapes)
        {
            crb200::setLastError("CrB200SolverSetNumShapes: at most 64 shapes per scene");
            return CRB200_ERR_CAPACITY;
        }
        s->numShapes = numShapes;
        s->configVersion++;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverBindShapeIds(CrB200SolverHandle solver, int *shapeIds)
    {
        SOLVER_OR_FAIL(solver);
        s->shapeIds = shapeIds;
        s->configVersion++;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverBindShapeData(CrB200SolverHandle solver, const CrB200ShapeData *shapes)
    {
        SOLVER_OR_FAIL(solver);
        if (!shapes)
            return bad("CrB200SolverBindShapeData: null pointer");
        s->shapes = *shapes;
        s->configVersion++;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverBindGeometryData(CrB200SolverHandle solver, const CrB200GeometryData *geometries)
    {
        SOLVER_OR_FAIL(solver);
        if (!geometries)
            return bad("CrB200SolverBindGeometryData: null pointer");
        s->geometries = *geometries;
        s->configVersion++;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverBindGeometrySdfData(CrB200SolverHandle solver, const CrB200GeometrySdfData *sdf)
    {
        SOLVER_OR_FAIL(solver);
        if (!sdf)
            return bad("CrB200SolverBindGeometrySdfData: null pointer");
        s->sdf = *sdf;
        s->configVersion++;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverGetGridDims(CrB200SolverHandle solver, int outDims[3])
    {
        SOLVER_OR_FAIL(solver);
        if (!outDims)
            return bad("CrB200SolverGetGridDims: null pointer");
        outDims[0] = s->geom.n.x;
        outDims[1] = s->geom.n.y;
        outDims[2] = s->geom.n.z;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverCopyParticleState(CrB200SolverHandle solver, unsigned int n, float *F, float *C,
                                                 float *V0)
    {
        SOLVER_OR_FAIL(solver);
        if (!s->initialized)
        {
            crb200::setLastError("CrB200SolverCopyParticleState: solver not initialized");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        if (n > (unsigned)s->numMaxParticles)
            return bad("CrB200SolverCopyParticleState: n exceeds numMaxParticles");
        if (int rc = s->residentSyncPlanes())
            return rc;
        const size_t stride = (size_t)s->numMaxParticles;
        // planes -> per-particle 9 floats: a strided 2D copy per matrix
        if (F)
        {
            for (int k = 0; k < 9; ++k)
            {
                cudaError_t e = cudaMemcpy2DAsync(F + k, 9 * sizeof(float), s->F + k * stride, sizeof(float), sizeof(float), n,
                                      cudaMemcpyDeviceToDevice, s->stream);
                if (e != cudaSuccess)
                    return crb200::cudaFail(e, "copy F");
            }
        }
        if (C)
            for (int k = 0; k < 9; ++k)
            {
                cudaError_t e = cudaMemcpy2DAsync(C + k, 9 * sizeof(float), s->Cm + k * stride, sizeof(float),
                                                  sizeof(float), n, cudaMemcpyDeviceToDevice, s->stream);
                if (e != cudaSuccess)
                    return crb200::cudaFail(e, "copy C");
            }
        if (V0)
        {
            cudaError_t e = cudaMemcpyAsync(V0, s->V0, n * sizeof(float), cudaMemcpyDeviceToDevice, s->stream);
            if (e != cudaSuccess)
                return crb200::cudaFail(e, "copy V0");
        }
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverSetParticleState(CrB200SolverHandle solver, unsigned int n, const float *F,
                                                const float *C, const float *V0)
    {
        SOLVER_OR_FAIL(solver);
        if (!s->initialized)
        {
            crb200::setLastError("CrB200SolverSetParticleState: solver not initialized");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        if (n > (unsigned)s->numMaxParticles)
            return bad("CrB200SolverSetParticleState: n exceeds numMaxParticles");
        if (int rc = s->residentRetire()) // the new state is read from the particle-id planes
            return rc;
        const size_t stride = (size_t)s->numMaxParticles;
        for (int k = 0; k < 9; ++k)
        {
            if (F)
            {
                cudaError_t e = cudaMemcpy2DAsync(s->F + k * stride, sizeof(float), F + k, 9 * sizeof(float),
                                                  sizeof(float), n, cudaMemcpyDeviceToDevice, s->stream);
                if (e != cudaSuccess)
                    return crb200::cudaFail(e, "set F");
            }
            if (C)
            {
                cudaError_t e = cudaMemcpy2DAsync(s->Cm + k * stride, sizeof(float), C + k, 9 * sizeof(float),
                                                  sizeof(float), n, cudaMemcpyDeviceToDevice, s->stream);
                if (e != cudaSuccess)
                    return crb200::cudaFail(e, "set C");
            }
        }
        if (V0)
        {
            cudaError_t e = cudaMemcpyAsync(s->V0, V0, n * sizeof(float), cudaMemcpyDeviceToDevice, s->stream);
            if (e != cudaSuccess)
                return crb200::cudaFail(e, "set V0");
        }
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverCopySortState(CrB200SolverHandle solver, unsigned int *keys, unsigned int *sortedIds,
                                             unsigned int *outNumSortedHost)
    {
        SOLVER_OR_FAIL(solver);
        if (!s->initialized)
        {
            crb200::setLastError("CrB200SolverCopySortState: solver not initialized");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        // a sort of the current positions, then its products
        if (keys || sortedIds)
        {
            const int r = s->copySortState(keys, sortedIds);
            if (r != CRB200_OK)
                return r;
        }
        crb200::SortHeader h;
        cudaError_t e = cudaMemcpyAsync(&h, s->header, sizeof(h), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess)
            return crb200::cudaFail(e, "read sort header");
        if (outNumSortedHost)
            *outNumSortedHost = h.numSorted;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverCopyCutMasks(CrB200SolverHandle solver, unsigned int *masks)
    {
        SOLVER_OR_FAIL(solver);
        if (!masks)
            return bad("CrB200SolverCopyCutMasks: null pointer");
        if (!s->initialized)
        {
            crb200::setLastError("CrB200SolverCopyCutMasks: solver not initialized");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        crb200::SortHeader h;
        cudaError_t e = cudaMemcpyAsync(&h, s->header, sizeof(h), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess)
            return crb200::cudaFail(e, "read shape flags");
        const unsigned n = s->totalParticles();
        if (s->resValid && s->numShapes > 0 && (h.shapeFlags & crb200::SF_SLICER))
            return s->copyCutMasks(masks); // the resident path keeps them in its slots
        if (s->numShapes == 0 || (!s->isBatch() && !(h.shapeFlags & crb200::SF_SLICER)))
            e = cudaMemsetAsync(masks, 0, n * sizeof(unsigned), s->stream); // nothing is cut
        else
            e = cudaMemcpyAsync(masks, s->cutMasks, n * sizeof(unsigned), cudaMemcpyDeviceToDevice, s->stream);
        return crb200::cudaFail(e, "copy cut masks");
    }

    CRB200_API int CrB200SolverGetStatus(CrB200SolverHandle solver, unsigned int *outStatusHost, int timeoutMs)
    {
        SOLVER_OR_FAIL(solver);
        if (!outStatusHost)
            return bad("CrB200SolverGetStatus: null pointer");
        if (!s->initialized)
        {
            *outStatusHost = 0;
            return CRB200_OK;
        }
        const auto t0 = std::chrono::steady_clock::now();
        for (;;)
        {
            cudaError_t q = cudaStreamQuery(s->stream);
            if (q == cudaSuccess)
                break;
            if (q != cudaErrorNotReady)
                return crb200::cudaFail(q, "cudaStreamQuery");
            if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(timeoutMs))
            {
                crb200::setLastError("CrB200SolverGetStatus: solver stream still busy");
                return CRB200_ERR_TIMEOUT;
            }
            std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
        crb200::SortHeader h;
        cudaError_t e = cudaMemcpy(&h, s->header, sizeof(h), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess)
            return crb200::cudaFail(e, "read status");
        *outStatusHost = h.status;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverClearStatus(CrB200SolverHandle solver)
    {
        SOLVER_OR_FAIL(solver);
        if (!s->initialized)
            return CRB200_OK;
        cudaError_t e = cudaMemsetAsync(&s->header->status, 0, sizeof(unsigned), s->stream);
        return crb200::cudaFail(e, "clear status");
    }

    CRB200_API int CrB200SolverSetOption(CrB200SolverHandle solver, int option, int value)
    {
        SOLVER_OR_FAIL(solver);
        if (option == CRB200_OPT_PHASE_TIMING)
            s->phaseTiming = value != 0;
        else if (option == CRB200_OPT_DETERMINISTIC_COUPLING)
        {
            if (int rc = s->setDeterministicCoupling(value != 0))
                return rc;
        }
        else if (option == CRB200_OPT_DETERMINISTIC)
        {
            if (int rc = s->setDeterministic(value != 0))
                return rc;
        }
        else if (option == CRB200_OPT_RESIDENT)
        {
            if (value == 0)
                if (int rc = s->residentRetire())
                    return rc;
            s->residentOn = value != 0;
        }
        else if (option == CRB200_OPT_STANDARD_GPU_SEMANTICS)
        {
            if (int rc = s->setStdGpuSemantics(value != 0))
                return rc;
        }
        else
            return bad("CrB200SolverSetOption: unknown option");
        s->configVersion++;
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverAdvance(CrB200SolverHandle solver, float dt, CrB200Float4 *positionMassHost,
                                       CrB200Float4 *velocityHost, int *outSubsteps)
    {
        SOLVER_OR_FAIL(solver);
        if (!s->initialized)
        {
            crb200::setLastError("CrB200SolverAdvance: solver not initialized");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        if (!(dt >= 0.f))
            return bad("CrB200SolverAdvance: dt must be non-negative");
        if (!(dt <= s->dt * 1.0e6f))
            return bad("CrB200SolverAdvance: dt spans more than a million substeps");
        return s->advance(dt, reinterpret_cast<float4 *>(positionMassHost), reinterpret_cast<float4 *>(velocityHost),
                          outSubsteps);
    }

    CRB200_API int CrB200SolverAdvanceAsync(CrB200SolverHandle solver, float dt, CrB200Float4 *positionMassHost,
                                            CrB200Float4 *velocityHost, int *outSubsteps)
    {
        SOLVER_OR_FAIL(solver);
        if (!s->initialized)
        {
            crb200::setLastError("CrB200SolverAdvanceAsync: solver not initialized");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        if (!(dt >= 0.f))
            return bad("CrB200SolverAdvanceAsync: dt must be non-negative");
        if (!(dt <= s->dt * 1.0e6f))
            return bad("CrB200SolverAdvanceAsync: dt spans more than a million substeps");
        return s->advanceAsync(dt, reinterpret_cast<float4 *>(positionMassHost),
                               reinterpret_cast<float4 *>(velocityHost), outSubsteps);
    }

    CRB200_API int CrB200SolverAutotune(CrB200SolverHandle solver, int substepsPerTrial, int *outChoiceHost)
    {
        SOLVER_OR_FAIL(solver);
        if (substepsPerTrial < 0)
            return bad("CrB200SolverAutotune: negative substep count");
        return s->autotune(substepsPerTrial, outChoiceHost);
    }

    CRB200_API int CrB200SolverAdjointRecord(CrB200SolverHandle solver, int numSubsteps, int checkpointInterval,
                                             int numCaptures, const int *captureSubsteps,
                                             CrB200Float4 *capturedPositions)
    {
        SOLVER_OR_FAIL(solver);
        if (numSubsteps <= 0 || checkpointInterval <= 0)
            return bad("CrB200SolverAdjointRecord: numSubsteps and checkpointInterval must be positive");
        if (numCaptures < 0 || (numCaptures > 0 && (!captureSubsteps || !capturedPositions)))
            return bad("CrB200SolverAdjointRecord: captures need a substep list and an output buffer");
        for (int i = 0; i < numCaptures; ++i)
        {
            const int t = captureSubsteps[i];
            if (t < 1 || t > numSubsteps || (i > 0 && t <= captureSubsteps[i - 1]))
                return bad("CrB200SolverAdjointRecord: capture substeps must increase strictly within [1, numSubsteps]");
        }
        return s->adjointRecord(numSubsteps, checkpointInterval, captureSubsteps, numCaptures,
                                reinterpret_cast<float4 *>(capturedPositions));
    }

    CRB200_API int CrB200SolverAdjointBackward(CrB200SolverHandle solver, const CrB200Float4 *gradPositions,
                                               CrB200Float4 *gradVelocity, CrB200Float4 *gradMaterial,
                                               CrB200Float4 *gradPosition)
    {
        SOLVER_OR_FAIL(solver);
        if (!gradPositions && !s->adjCaptures.empty())
            return bad("CrB200SolverAdjointBackward: null gradPositions");
        return s->adjointBackward(reinterpret_cast<const float4 *>(gradPositions), reinterpret_cast<float4 *>(gradVelocity),
                                  reinterpret_cast<float4 *>(gradMaterial), reinterpret_cast<float4 *>(gradPosition));
    }

    CRB200_API int CrB200SolverGetPhaseTimes(CrB200SolverHandle solver, float outMs[CRB200_NUM_PHASES],
                                             int *outSubsteps, int reset)
    {
        SOLVER_OR_FAIL(solver);
        if (!outMs)
            return bad("CrB200SolverGetPhaseTimes: null pointer");
        cudaError_t e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess)
            return crb200::cudaFail(e, "phase times");
        for (int k = 0; k < CRB200_NUM_PHASES; ++k)
            outMs[k] = s->phaseMs[k];
        if (outSubsteps)
            *outSubsteps = s->phaseSteps;
        if (reset)
        {
            for (int k = 0; k < CRB200_NUM_PHASES; ++k)
                s->phaseMs[k] = 0.f;
            s->phaseSteps = 0;
        }
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverGetResidentKernelTime(CrB200SolverHandle solver, float *outMs, int *outLaunches,
                                                     int reset)
    {
        SOLVER_OR_FAIL(solver);
        if (!outMs || !outLaunches)
            return bad("CrB200SolverGetResidentKernelTime: null pointer");
        cudaError_t e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess)
            return crb200::cudaFail(e, "resident kernel time");
        *outMs = s->fusedMs;
        *outLaunches = s->fusedLaunches;
        if (reset)
        {
            s->fusedMs = 0.f;
            s->fusedLaunches = 0;
        }
        return CRB200_OK;
    }

    CRB200_API int CrB200SolverGetFp64Fallbacks(CrB200SolverHandle solver, unsigned int *outCountHost, int reset)
    {
        SOLVER_OR_FAIL(solver);
        if (!outCountHost)
            return bad("CrB200SolverGetFp64Fallbacks: null pointer");
        if (!s->initialized)
        {
            *outCountHost = 0;
            return CRB200_OK;
        }
        cudaError_t e = cudaMemcpyAsync(outCountHost, &s->header->fp64Fallbacks, sizeof(unsigned),
                                        cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(s->stream);
        if (e == cudaSuccess && reset)
            e = cudaMemsetAsync(&s->header->fp64Fallbacks, 0, sizeof(unsigned), s->stream);
        return crb200::cudaFail(e, "fp64 fallback count");
    }

    CRB200_API int CrB200SvdBatch(unsigned int n, const float *A, float *U, float *V, float *S, float *R,
                                  unsigned int *fp64Used, unsigned int *fp64Count, void *stream)
    {
        if (n > 0 && (!A || !U || !V || !S || !R || !fp64Used))
            return bad("CrB200SvdBatch: null array");
        return crb200::svdBatch(n, A, U, V, S, R, fp64Used, fp64Count, static_cast<cudaStream_t>(stream));
    }

    CRB200_API int CrB200SolverGetGridStats(CrB200SolverHandle solver, unsigned int outStats[4])
    {
        SOLVER_OR_FAIL(solver);
        if (!outStats)
            return bad("CrB200SolverGetGridStats: null pointer");
        if (!s->initialized)
        {
            crb200::setLastError("CrB200SolverGetGridStats: solver not initialized");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        crb200::SortHeader h;
        cudaError_t e = cudaMemcpyAsync(&h, s->header, sizeof(h), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess)
            return crb200::cudaFail(e, "grid stats");
        outStats[0] = h.numSorted;
        outStats[1] = h.numActiveBlocks;
        outStats[2] = h.numTouchedBlocks;
        outStats[3] = h.touchedNodes;
        return CRB200_OK;
    }
}
