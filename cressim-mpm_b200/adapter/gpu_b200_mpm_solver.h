// Drop-in solver for CRESSim-MPM: a MpmSolverGpu (src/solver/mpm_solver_gpu.h:43-57) whose every
// MpmSolver member (include/solver/mpm_solver.h:63-191) forwards to libcrmpm_b200.so.
//
// This header is compiled inside the reference's engine target: it includes
// the reference's own solver headers, and SimulationFactoryImpl::createScene
// (src/engine/simulation_factory_impl.cpp:296-349) constructs it in place of GpuMlsMpmSolver,
// GpuPbMpmSolver or GpuStandardMpmSolver.  The factory sets the CUDA stream before initialize()
// (:341-349) and SceneImpl binds particle data before initialize() (src/engine/scene_impl.cpp:42-93);
// counts and shape bindings that change later (setNumActiveParticles, setNumShapes, bindShapeIds)
// are compared with what the engine holds at every step(), as the reference's solvers read them
// at every launch, and only changed ones cross the C ABI.  Errors are logged the way the
// reference logs CUDA errors and execution continues.
//
// GpuB200MlsMpmSolver, GpuB200PbMpmSolver and GpuB200StandardMpmSolver take the constructor
// arguments of GpuMlsMpmSolver, GpuPbMpmSolver and GpuStandardMpmSolver, so the switch in
// createScene changes only the class names.
#ifndef CR_GPU_B200_MPM_SOLVER_H
#define CR_GPU_B200_MPM_SOLVER_H

#include <cstdio>
#include <cstring>

#include "crmpm_b200.h"
#include "mpm_solver_gpu.h"

namespace crmpm
{
    class GpuB200MpmSolver : public MpmSolverGpu
    {
    public:
        // solverType: MpmSolverType::eGpuMlsMpmSolver, eGpuPbMpmSolver or eGpuStandardMpmSolver.
        GpuB200MpmSolver(MpmSolverType solverType, int numParticles, float cellSize, Bounds3 gridBound)
            : mType(static_cast<int>(solverType)), mCellSize(cellSize)
        {
            mNumMaxParticles = numParticles;
            mGridBound = gridBound;
        }

        void initialize() override
        {
            const float mn[3] = {mGridBound.minimum.x(), mGridBound.minimum.y(), mGridBound.minimum.z()};
            const float mx[3] = {mGridBound.maximum.x(), mGridBound.maximum.y(), mGridBound.maximum.z()};
            check(CrB200SolverCreate(mType, mNumMaxParticles, mCellSize, mn, mx, mCudaStream, &mHandle));
            // inactive particles of standard MPM as GpuStandardMpmSolver treats them
            if (mType == static_cast<int>(MpmSolverType::eGpuStandardMpmSolver))
                check(CrB200SolverSetOption(mHandle, CRB200_OPT_STANDARD_GPU_SEMANTICS, 1));
            check(CrB200SolverBindParticleData(mHandle, reinterpret_cast<CrB200Float4 *>(mParticleData->positionMass),
                                               reinterpret_cast<CrB200Float4 *>(mParticleData->velocity)));
            check(CrB200SolverBindParticleMaterials(mHandle,
                                                    reinterpret_cast<CrB200Float4 *>(mParticleMaterialData->params0),
                                                    reinterpret_cast<int *>(mParticleMaterialData->type)));
            check(CrB200SolverBindActiveMask(mHandle, mActiveMask));
            pushState();
            check(CrB200SolverInitialize(mHandle));
        }

        float step() override
        {
            pushState();
            check(CrB200SolverStep(mHandle, nullptr));
            return mIntegrationStepSize;
        }

        // Calls of the C ABI made by step() since the solver was made (the fixed cost a substep
        // adds on the host); every one but the step itself is a changed setting.
        unsigned long long abiCalls() const { return mAbiCalls; }

        void computeInitialData(unsigned int numParticlesToCompute, const unsigned int *CR_RESTRICT indices) override
        {
            check(CrB200SolverComputeInitialData(mHandle, numParticlesToCompute, indices));
        }

        void setSolverIterations(int n) override { mIterations = n; }

    protected:
        void _release() override
        {
            if (mHandle)
                check(CrB200SolverRelease(mHandle));
            mHandle = nullptr;
        }

        // The engine runs the whole substep in step(); the staged hooks of MpmSolverBase are unused.
        void resetGrid() override {}
        void particleToGrid() override {}
        void updateGrid() override {}
        void gridToParticle() override {}

    private:
        int mType;
        float mCellSize;
        int mIterations = 10; // GpuPbMpmSolver default (gpu_pb_mpm_solver.cuh:53)
        CrB200SolverHandle mHandle = nullptr;

        // What the engine was last given (pushState sends only what differs).
        struct Pushed
        {
            bool valid = false;
            float g[3] = {0.f, 0.f, 0.f};
            float dt = 0.f;
            int iterations = 0, contactModel = 0, numShapes = 0;
            unsigned numActive = 0;
            const int *shapeIds = nullptr;
            // the descriptors are compared by content: the factory regrows the arrays they point
            // to in place of the old ones without moving the descriptors themselves
            CrB200ShapeData shapeData{};
            CrB200GeometryData geometryData{};
            CrB200GeometrySdfData sdfData{};
        } mPushed;
        unsigned long long mAbiCalls = 0;

        void pushState()
        {
            Pushed &q = mPushed;
            const Vec3f &g = mGravity;
            const bool all = !q.valid;
            if (all || q.g[0] != g.data.x || q.g[1] != g.data.y || q.g[2] != g.data.z)
            {
                check(CrB200SolverSetGravity(mHandle, g.data.x, g.data.y, g.data.z));
                q.g[0] = g.data.x;
                q.g[1] = g.data.y;
                q.g[2] = g.data.z;
            }
            if (all || q.dt != mIntegrationStepSize)
            {
                check(CrB200SolverSetIntegrationStepSize(mHandle, mIntegrationStepSize));
                q.dt = mIntegrationStepSize;
            }
            if (all || q.iterations != mIterations)
            {
                check(CrB200SolverSetSolverIterations(mHandle, mIterations));
                q.iterations = mIterations;
            }
            const int cm = static_cast<int>(mShapeContactModel);
            if (all || q.contactModel != cm)
            {
                check(CrB200SolverSetShapeContactModel(mHandle, cm));
                q.contactModel = cm;
            }
            if (all || q.numActive != mNumActiveParticles)
            {
                check(CrB200SolverSetNumActiveParticles(mHandle, mNumActiveParticles));
                q.numActive = mNumActiveParticles;
            }
            if (all || q.numShapes != mNumShapes)
            {
                check(CrB200SolverSetNumShapes(mHandle, mNumShapes));
                q.numShapes = mNumShapes;
            }
            if (mNumShapes > 0)
            {
                if (all || q.shapeIds != mShapeIds)
                {
                    check(CrB200SolverBindShapeIds(mHandle, mShapeIds));
                    q.shapeIds = mShapeIds;
                }
                const auto *sd = reinterpret_cast<const CrB200ShapeData *>(mShapeData);
                if (all || std::memcmp(&q.shapeData, sd, sizeof(*sd)) != 0)
                {
                    check(CrB200SolverBindShapeData(mHandle, sd));
                    q.shapeData = *sd;
                }
                const auto *gd = reinterpret_cast<const CrB200GeometryData *>(mGeometryData);
                if (all || std::memcmp(&q.geometryData, gd, sizeof(*gd)) != 0)
                {
                    check(CrB200SolverBindGeometryData(mHandle, gd));
                    q.geometryData = *gd;
                }
                const auto *fd = reinterpret_cast<const CrB200GeometrySdfData *>(mGeometrySdfData);
                if (all || std::memcmp(&q.sdfData, fd, sizeof(*fd)) != 0)
                {
                    check(CrB200SolverBindGeometrySdfData(mHandle, fd));
                    q.sdfData = *fd;
                }
            }
            q.valid = true;
        }

        void check(int rc)
        {
            ++mAbiCalls;
            if (rc != CRB200_OK)
                std::fprintf(stderr, "crmpm_b200 error %d: %s\n", rc, CrB200GetLastError());
        }

        static_assert(sizeof(ShapeData) == sizeof(CrB200ShapeData), "ShapeData layout");
        static_assert(sizeof(GeometryData) == sizeof(CrB200GeometryData), "GeometryData layout");
        static_assert(sizeof(GeometrySdfData) == sizeof(CrB200GeometrySdfData), "GeometrySdfData layout");
        static_assert(sizeof(Vec3f) == sizeof(CrB200Float4) && sizeof(Quat) == sizeof(CrB200Float4), "float4 layout");
        static_assert(sizeof(ParticleMaterialType) == sizeof(int), "material type layout");
    };

    // The solver classes createScene constructs (simulation_factory_impl.cpp:306-333), with their
    // constructor arguments, each running the engine in the matching mode.
    class GpuB200MlsMpmSolver : public GpuB200MpmSolver
    {
    public:
        GpuB200MlsMpmSolver(int numParticles, float cellSize, Bounds3 gridBound)
            : GpuB200MpmSolver(MpmSolverType::eGpuMlsMpmSolver, numParticles, cellSize, gridBound) {}
    };
    class GpuB200PbMpmSolver : public GpuB200MpmSolver
    {
    public:
        GpuB200PbMpmSolver(int numParticles, float cellSize, Bounds3 gridBound)
            : GpuB200MpmSolver(MpmSolverType::eGpuPbMpmSolver, numParticles, cellSize, gridBound) {}
    };
    class GpuB200StandardMpmSolver : public GpuB200MpmSolver
    {
    public:
        GpuB200StandardMpmSolver(int numParticles, float cellSize, Bounds3 gridBound)
            : GpuB200MpmSolver(MpmSolverType::eGpuStandardMpmSolver, numParticles, cellSize, gridBound) {}
    };
} // namespace crmpm

#endif // !CR_GPU_B200_MPM_SOLVER_H
