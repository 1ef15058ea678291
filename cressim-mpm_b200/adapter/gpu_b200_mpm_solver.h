// Drop-in solver for CRESSim-MPM: a MpmSolverGpu (src/solver/mpm_solver_gpu.h:43-57) whose every
// MpmSolver member (include/solver/mpm_solver.h:63-191) forwards to libcrmpm_b200.so.
//
// This header is compiled inside the reference's engine target: it includes
// the reference's own solver headers, and SimulationFactoryImpl::createScene
// (src/engine/simulation_factory_impl.cpp:296-349) constructs it in place of GpuMlsMpmSolver,
// GpuPbMpmSolver or GpuStandardMpmSolver.  The factory sets the CUDA stream before initialize()
// (:341-349) and SceneImpl binds particle data before initialize() (src/engine/scene_impl.cpp:42-93);
// counts and shape bindings that change later (setNumActiveParticles, setNumShapes, bindShapeIds)
// are pushed to the engine at every step(), as the reference's solvers read them at every launch.
// Errors are logged the way the reference logs CUDA errors and execution continues.
#ifndef CR_GPU_B200_MPM_SOLVER_H
#define CR_GPU_B200_MPM_SOLVER_H

#include <cstdio>

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

        void pushState()
        {
            const Vec3f &g = mGravity;
            check(CrB200SolverSetGravity(mHandle, g.data.x, g.data.y, g.data.z));
            check(CrB200SolverSetIntegrationStepSize(mHandle, mIntegrationStepSize));
            check(CrB200SolverSetSolverIterations(mHandle, mIterations));
            check(CrB200SolverSetShapeContactModel(mHandle, static_cast<int>(mShapeContactModel)));
            check(CrB200SolverSetNumActiveParticles(mHandle, mNumActiveParticles));
            check(CrB200SolverSetNumShapes(mHandle, mNumShapes));
            if (mNumShapes > 0)
            {
                check(CrB200SolverBindShapeIds(mHandle, mShapeIds));
                check(CrB200SolverBindShapeData(mHandle, reinterpret_cast<const CrB200ShapeData *>(mShapeData)));
                check(CrB200SolverBindGeometryData(mHandle, reinterpret_cast<const CrB200GeometryData *>(mGeometryData)));
                check(CrB200SolverBindGeometrySdfData(mHandle,
                                                      reinterpret_cast<const CrB200GeometrySdfData *>(mGeometrySdfData)));
            }
        }

        static void check(int rc)
        {
            if (rc != CRB200_OK)
                std::fprintf(stderr, "crmpm_b200 error %d: %s\n", rc, CrB200GetLastError());
        }

        static_assert(sizeof(ShapeData) == sizeof(CrB200ShapeData), "ShapeData layout");
        static_assert(sizeof(GeometryData) == sizeof(CrB200GeometryData), "GeometryData layout");
        static_assert(sizeof(GeometrySdfData) == sizeof(CrB200GeometrySdfData), "GeometrySdfData layout");
        static_assert(sizeof(Vec3f) == sizeof(CrB200Float4) && sizeof(Quat) == sizeof(CrB200Float4), "float4 layout");
        static_assert(sizeof(ParticleMaterialType) == sizeof(int), "material type layout");
    };
} // namespace crmpm

#endif // !CR_GPU_B200_MPM_SOLVER_H
