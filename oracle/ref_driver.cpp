// ORACLE / TEST INFRASTRUCTURE ONLY.  Never linked into, loaded by, or called from the product.
//
// Host driver around CRESSim-MPM's own header-only substep algorithms.  It is compiled by
// oracle/Makefile against the reference sources where they lie and written to oracle/_ref/;
// nothing of the reference is copied here.  The loops below restate the orchestration of the
// reference's single-threaded CPU solvers, which call the very same headers the GPU solvers call:
//   MLS-MPM   src/solver/cpu_mls_mpm_solver.cpp:60-210
//   PB-MPM    src/solver/cpu_pb_mpm_solver.cpp:96-236
//   standard  src/solver/cpu_standard_mpm_solver.cpp:50-197
// so its outputs are the reference's own arithmetic, in the reference's own (serial) order.
//
// Build flags (-ffp-contract=off, no -ffast-math) keep the host arithmetic IEEE single precision
// with no fused multiply-add, which is what the reference's CPU build produces on x86-64.

#include <cstdint>
#include <cstring>
#include <vector>

#include "mls_mpm_algorithm.h"
#include "pb_mpm_algorithm.h"
#include "standard_mpm_algorithm.h"

#include "crmpm_b200.h"

using namespace crmpm;

namespace
{
    struct RefSolver
    {
        int solverType;
        int numMaxParticles;
        Bounds3 bound;
        float cellSize, invCellSize, cellVolume;
        Vec3i numNodesPerDim;
        int numNodes;

        float dt = 0.002f;
        Vec3f gravity;
        int iterations = 10;
        int contactModel = 0;

        float4 *positionMass = nullptr;
        Vec3f *velocity = nullptr;
        float4 *matParams = nullptr;
        ParticleMaterialType *matType = nullptr;
        unsigned char *mask = nullptr;
        unsigned int numActive = 0;

        std::vector<float> V0;
        std::vector<Mat3x3f> F, C;
        std::vector<float4> grid;
        std::vector<Vec3f> force;

        int numShapes = 0;
        int *shapeIds = nullptr;
        ShapeData shapes{};
        GeometryData geoms{};
        GeometrySdfData sdf{};
    };

    // Constructor arithmetic of every reference solver (gpu_mls_mpm_solver.cu:40-52,
    // cpu_mls_mpm_solver.cpp:39-51): node counts are int((max - min) / dx + 1) in float.
    void setupGrid(RefSolver &s, float cellSize, const float mn[3], const float mx[3])
    {
        s.bound = Bounds3(Vec3f(mn[0], mn[1], mn[2]), Vec3f(mx[0], mx[1], mx[2]));
        s.cellSize = cellSize;
        s.invCellSize = 1 / cellSize;
        Vec3f gridSize = s.bound.maximum - s.bound.minimum;
        s.numNodesPerDim = (gridSize / cellSize + 1.0f).cast<int>();
        s.numNodes = s.numNodesPerDim.x() * s.numNodesPerDim.y() * s.numNodesPerDim.z();
        s.cellVolume = cellSize * cellSize * cellSize;
    }

    void resetGrid(RefSolver &s)
    {
        for (int i = 0; i < s.numNodes; ++i)
            s.grid[i] = make_float4(0, 0, 0, 0);
        if (s.solverType == CRB200_SOLVER_GPU_STANDARD)
            for (int i = 0; i < s.numNodes; ++i)
                s.force[i] = Vec3f(0, 0, 0);
    }

    // ---------------- MLS-MPM: cpu_mls_mpm_solver.cpp:95-210 ----------------
    void mlsP2G(RefSolver &s)
    {
        for (int idx = 0; idx < (int)s.numActive; ++idx)
        {
            if (!s.mask[idx])
                continue;
            mlsMpmParticleToGrid<false>(s.dt, s.gravity, s.bound.minimum, s.invCellSize, s.cellSize,
                                        s.numNodesPerDim, s.positionMass[idx], s.V0[idx], s.F[idx], s.C[idx],
                                        s.matParams[idx], s.matType[idx], s.numShapes, s.shapeIds, s.shapes,
                                        s.geoms, s.sdf, s.velocity[idx], s.grid.data());
        }
    }

    void mlsUpdate(RefSolver &s)
    {
        for (int n = 0; n < s.numNodes; ++n)
        {
            if (s.contactModel == 0)
                mlsMpmUpdateGrid<false, false>(s.dt, n, s.bound.minimum, s.cellSize, s.numNodesPerDim,
                                               s.numShapes, s.shapeIds, s.shapes, s.geoms, s.sdf, s.grid.data());
            else
                mlsMpmUpdateGrid<false, true>(s.dt, n, s.bound.minimum, s.cellSize, s.numNodesPerDim,
                                              s.numShapes, s.shapeIds, s.shapes, s.geoms, s.sdf, s.grid.data());
        }
    }

    void mlsG2P(RefSolver &s)
    {
        for (int idx = 0; idx < (int)s.numActive; ++idx)
        {
            if (!s.mask[idx])
                continue;
            mlsMpmGridToParticle<false>(s.bound.minimum, s.bound.maximum, s.invCellSize, s.cellSize,
                                        s.numNodesPerDim, s.dt, s.grid.data(), s.numShapes, s.shapeIds,
                                        s.shapes, s.geoms, s.sdf, s.positionMass[idx], s.velocity[idx],
                                        s.F[idx], s.C[idx]);
        }
    }

    // ---------------- PB-MPM: cpu_pb_mpm_solver.cpp:96-236 ----------------
    void pbP2G(RefSolver &s)
    {
        for (int idx = 0; idx < (int)s.numActive; ++idx)
        {
            if (!s.mask[idx])
                continue;
            pbMpmParticleToGrid<false>(s.dt, s.bound.minimum, s.invCellSize, s.cellSize, s.numNodesPerDim,
                                       s.positionMass[idx], s.velocity[idx], s.F[idx], s.matParams[idx],
                                       s.matType[idx], s.numShapes, s.shapeIds, s.shapes, s.geoms, s.sdf,
                                       s.C[idx], s.grid.data());
        }
    }

    void pbUpdate(RefSolver &s)
    {
        for (int n = 0; n < s.numNodes; ++n)
        {
            if (s.contactModel == 0)
                pbMpmUpdateGrid<false, false>(s.dt, n, s.bound.minimum, s.cellSize, s.numNodesPerDim,
                                              s.numShapes, s.shapeIds, s.shapes, s.geoms, s.sdf, s.grid.data());
            else
                pbMpmUpdateGrid<false, true>(s.dt, n, s.bound.minimum, s.cellSize, s.numNodesPerDim,
                                             s.numShapes, s.shapeIds, s.shapes, s.geoms, s.sdf, s.grid.data());
        }
    }

    void pbG2P(RefSolver &s)
    {
        for (int idx = 0; idx < (int)s.numActive; ++idx)
        {
            if (!s.mask[idx])
                continue;
            pbMpmGridToParticle(s.bound.minimum, s.bound.maximum, s.invCellSize, s.cellSize, s.cellVolume,
                                s.numNodesPerDim, s.dt, s.grid.data(), s.numShapes, s.shapeIds, s.shapes,
                                s.geoms, s.sdf, s.positionMass[idx], s.velocity[idx], s.C[idx]);
        }
    }

    void pbIntegrate(RefSolver &s)
    {
        for (int idx = 0; idx < (int)s.numActive; ++idx)
        {
            if (!s.mask[idx])
                continue;
            pbMpmIntegrateParticle<false>(s.bound.minimum, s.bound.maximum, s.dt, s.gravity, s.C[idx],
                                          s.matType[idx], s.numShapes, s.shapeIds, s.shapes, s.geoms, s.sdf,
                                          s.positionMass[idx], s.velocity[idx], s.F[idx]);
        }
    }

    // ---------------- standard MPM: cpu_standard_mpm_solver.cpp:105-197 ----------------
    // (its P2G visits every index below numActive regardless of the mask; G2P honours the mask)
    void stdP2G(RefSolver &s)
    {
        for (int idx = 0; idx < (int)s.numActive; ++idx)
        {
            standardMpmParticleToGrid<false>(s.gravity, s.bound.minimum, s.invCellSize, s.numNodesPerDim,
                                             s.positionMass[idx], s.velocity[idx], s.V0[idx], s.F[idx],
                                             s.matParams[idx], s.matType[idx], s.grid.data(), s.force.data());
        }
    }

    void stdUpdate(RefSolver &s)
    {
        for (int n = 0; n < s.numNodes; ++n)
        {
            if (s.contactModel == 0)
                standardMpmUpdateGrid<false, false>(n, s.bound.minimum, s.cellSize, s.numNodesPerDim, s.dt,
                                                    s.force.data(), s.numShapes, s.shapeIds, s.shapes, s.geoms,
                                                    s.sdf, s.grid.data());
            else
                standardMpmUpdateGrid<false, true>(n, s.bound.minimum, s.cellSize, s.numNodesPerDim, s.dt,
                                                   s.force.data(), s.numShapes, s.shapeIds, s.shapes, s.geoms,
                                                   s.sdf, s.grid.data());
        }
    }

    void stdG2P(RefSolver &s)
    {
        for (int idx = 0; idx < (int)s.numActive; ++idx)
        {
            if (!s.mask[idx])
                continue;
            standardMpmGridToParticle<false>(s.bound.minimum, s.bound.maximum, s.invCellSize, s.numNodesPerDim,
                                             s.dt, s.grid.data(), s.numShapes, s.shapeIds, s.shapes, s.geoms,
                                             s.sdf, s.positionMass[idx], s.velocity[idx], s.F[idx]);
        }
    }
} // namespace

extern "C"
{
    void *ref_create(int solverType, int numMaxParticles, float cellSize, const float *mn, const float *mx)
    {
        RefSolver *s = new RefSolver();
        s->solverType = solverType;
        s->numMaxParticles = numMaxParticles;
        setupGrid(*s, cellSize, mn, mx);
        s->V0.assign(numMaxParticles, 0.0f);
        s->F.assign(numMaxParticles, Mat3x3f());
        s->C.assign(numMaxParticles, Mat3x3f());
        s->grid.assign(s->numNodes, make_float4(0, 0, 0, 0));
        if (solverType == CRB200_SOLVER_GPU_STANDARD)
            s->force.assign(s->numNodes, Vec3f(0, 0, 0));
        return s;
    }

    void ref_destroy(void *h) { delete static_cast<RefSolver *>(h); }

    void ref_grid_dims(void *h, int *out)
    {
        RefSolver &s = *static_cast<RefSolver *>(h);
        out[0] = s.numNodesPerDim.x();
        out[1] = s.numNodesPerDim.y();
        out[2] = s.numNodesPerDim.z();
    }

    void ref_set_params(void *h, float dt, const float *g, int iterations, int contactModel)
    {
        RefSolver &s = *static_cast<RefSolver *>(h);
        s.dt = dt;
        s.gravity = Vec3f(g[0], g[1], g[2]);
        s.iterations = iterations;
        s.contactModel = contactModel;
    }

    // Host arrays owned by the caller; layouts as in crmpm_b200.h.
    void ref_bind_particles(void *h, float *positionMass, float *velocity, float *matParams, int *matType,
                            unsigned char *mask, unsigned int numActive)
    {
        RefSolver &s = *static_cast<RefSolver *>(h);
        s.positionMass = reinterpret_cast<float4 *>(positionMass);
        s.velocity = reinterpret_cast<Vec3f *>(velocity);
        s.matParams = reinterpret_cast<float4 *>(matParams);
        s.matType = reinterpret_cast<ParticleMaterialType *>(matType);
        s.mask = mask;
        s.numActive = numActive;
    }

    void ref_bind_shapes(void *h, int numShapes, int *shapeIds, const CrB200ShapeData *shapes,
                         const CrB200GeometryData *geoms, const CrB200GeometrySdfData *sdf)
    {
        RefSolver &s = *static_cast<RefSolver *>(h);
        static_assert(sizeof(ShapeData) == sizeof(CrB200ShapeData), "ShapeData layout");
        static_assert(sizeof(GeometryData) == sizeof(CrB200GeometryData), "GeometryData layout");
        static_assert(sizeof(GeometrySdfData) == sizeof(CrB200GeometrySdfData), "GeometrySdfData layout");
        s.numShapes = numShapes;
        s.shapeIds = shapeIds;
        std::memcpy(&s.shapes, shapes, sizeof(ShapeData));
        std::memcpy(&s.geoms, geoms, sizeof(GeometryData));
        std::memcpy(&s.sdf, sdf, sizeof(GeometrySdfData));
    }

    // cpu_mls_mpm_solver.cpp:63-96 (the PB and standard solvers are identical in structure).
    // Like the reference it scatters into the live grid without clearing it first.
    void ref_compute_initial_data(void *h, unsigned int n, const unsigned int *indices)
    {
        RefSolver &s = *static_cast<RefSolver *>(h);
        for (unsigned int i = 0; i < n; ++i)
        {
            unsigned int idx = indices[i];
            s.F[idx].setIdentity();
            mlsMpmComputeInitialGridMass<false>(s.bound.minimum, s.invCellSize, s.numNodesPerDim, s.cellVolume,
                                                s.positionMass[idx], s.grid.data());
        }
        for (unsigned int i = 0; i < n; ++i)
        {
            unsigned int idx = indices[i];
            mlsMpmComputeInitialVolume(s.bound.minimum, s.invCellSize, s.numNodesPerDim, s.cellVolume,
                                       s.positionMass[idx], s.grid.data(), s.V0[idx]);
        }
    }

    // One reference step() (cpu_*_mpm_solver.cpp step()).
    void ref_step(void *h)
    {
        RefSolver &s = *static_cast<RefSolver *>(h);
        if (s.solverType == CRB200_SOLVER_GPU_MLS)
        {
            resetGrid(s);
            mlsP2G(s);
            mlsUpdate(s);
            mlsG2P(s);
        }
        else if (s.solverType == CRB200_SOLVER_GPU_PB)
        {
            for (int i = 0; i < s.iterations; i++)
            {
                resetGrid(s);
                pbP2G(s);
                pbUpdate(s);
                pbG2P(s);
            }
            pbIntegrate(s);
        }
        else
        {
            resetGrid(s);
            stdP2G(s);
            stdUpdate(s);
            stdG2P(s);
        }
    }

    // Single phases for operator-level tests: 0 reset, 1 P2G, 2 grid update, 3 G2P, 4 PB integrate.
    void ref_phase(void *h, int phase)
    {
        RefSolver &s = *static_cast<RefSolver *>(h);
        const bool mls = s.solverType == CRB200_SOLVER_GPU_MLS, pb = s.solverType == CRB200_SOLVER_GPU_PB;
        switch (phase)
        {
        case 0: resetGrid(s); break;
        case 1: mls ? mlsP2G(s) : pb ? pbP2G(s) : stdP2G(s); break;
        case 2: mls ? mlsUpdate(s) : pb ? pbUpdate(s) : stdUpdate(s); break;
        case 3: mls ? mlsG2P(s) : pb ? pbG2P(s) : stdG2P(s); break;
        case 4: if (pb) pbIntegrate(s); break;
        }
    }

    // F, C as float[n*9] column-major per particle; V0 float[n].
    void ref_get_state(void *h, unsigned int n, float *F9, float *C9, float *V0)
    {
        RefSolver &s = *static_cast<RefSolver *>(h);
        for (unsigned int p = 0; p < n; ++p)
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 3; ++r)
                {
                    if (F9) F9[p * 9 + c * 3 + r] = s.F[p](r, c);
                    if (C9) C9[p * 9 + c * 3 + r] = s.C[p](r, c);
                }
        if (V0)
            for (unsigned int p = 0; p < n; ++p)
                V0[p] = s.V0[p];
    }

    void ref_set_state(void *h, unsigned int n, const float *F9, const float *C9, const float *V0)
    {
        RefSolver &s = *static_cast<RefSolver *>(h);
        for (unsigned int p = 0; p < n; ++p)
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 3; ++r)
                {
                    if (F9) s.F[p](r, c) = F9[p * 9 + c * 3 + r];
                    if (C9) s.C[p](r, c) = C9[p * 9 + c * 3 + r];
                }
        if (V0)
            for (unsigned int p = 0; p < n; ++p)
                s.V0[p] = V0[p];
    }

    // Dense grid (float4 per node, x fastest) and, for standard MPM, the node force.
    void ref_get_grid(void *h, float *out4, float *force4)
    {
        RefSolver &s = *static_cast<RefSolver *>(h);
        std::memcpy(out4, s.grid.data(), sizeof(float4) * s.numNodes);
        if (force4 && !s.force.empty())
            std::memcpy(force4, s.force.data(), sizeof(float4) * s.numNodes);
    }

    void ref_set_grid(void *h, const float *in4)
    {
        RefSolver &s = *static_cast<RefSolver *>(h);
        std::memcpy(s.grid.data(), in4, sizeof(float4) * s.numNodes);
    }

    // Slicer masks with the reference's own predicate (mpm_rigid_contact.h:401-478) evaluated for
    // every stencil node exactly as MLS P2G does (mls_mpm_algorithm.h:166-211): bit i*9+j*3+k.
    void ref_cut_masks(void *h, unsigned int *out)
    {
        RefSolver &s = *static_cast<RefSolver *>(h);
        for (int idx = 0; idx < (int)s.numActive; ++idx)
        {
            unsigned int m = 0;
            const float4 &p = s.positionMass[idx];
            const Vec3f scaledPos = (p - s.bound.minimum) * s.invCellSize;
            const Vec3i baseCoord = (scaledPos - Vec3f(0.5f)).cast<int>();
            const Vec3f fx = scaledPos - baseCoord.cast<float>();
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++)
                    for (int k = 0; k < 3; k++)
                    {
                        Vec3i nodeCoord = baseCoord + Vec3i(i, j, k);
                        if (nodeCoord.x() < 0 || nodeCoord.x() >= s.numNodesPerDim.x() || nodeCoord.y() < 0 ||
                            nodeCoord.y() >= s.numNodesPerDim.y() || nodeCoord.z() < 0 ||
                            nodeCoord.z() >= s.numNodesPerDim.z())
                            continue;
                        const Vec3f d = (Vec3f(i, j, k) - fx) * s.cellSize;
                        if (checkOnDifferentSides<false>(p, (p + d).data, s.numShapes, s.shapeIds, s.shapes, s.geoms,
                                                         s.sdf))
                            m |= 1u << (i * 9 + j * 3 + k);
                    }
            out[idx] = m;
        }
    }

    // getGeometrySdf (sdf.h:67-496) at local points, for SDF unit tests.  out: float4 per point
    // (gradient, distance); tangent: float4 per point; spine: int per point.
    void ref_sdf_query(int geomType, const float *params0, const CrB200GeometrySdfData *sdfData, int n,
                       const float *localPts4, float *out4, float *tangent4, int *spine)
    {
        GeometrySdfData sd;
        std::memcpy(&sd, sdfData, sizeof(sd));
        float4 p0 = make_float4(params0[0], params0[1], params0[2], params0[3]);
        for (int i = 0; i < n; ++i)
        {
            Vec3f lp(localPts4[4 * i], localPts4[4 * i + 1], localPts4[4 * i + 2]);
            float4 r = make_float4(0, 0, 0, 0);
            Vec3f t;
            bool sp = getGeometrySdf(lp, (GeometryType)geomType, p0, sd.dimemsion, sd.lowerBoundCellSize,
                                     sd.gradientSignedDistance, r, &t);
            std::memcpy(out4 + 4 * i, &r, sizeof(float4));
            tangent4[4 * i] = t.x();
            tangent4[4 * i + 1] = t.y();
            tangent4[4 * i + 2] = t.z();
            tangent4[4 * i + 3] = 0;
            spine[i] = sp ? 1 : 0;
        }
    }

    // svd3 (include/math/svd3.h:1265-1276) on n column-major 3x3 matrices: U, Vt, sigma(3).
    void ref_svd3(int n, const float *A9, float *U9, float *Vt9, float *S3)
    {
        for (int p = 0; p < n; ++p)
        {
            Mat3x3f a;
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 3; ++r)
                    a(r, c) = A9[p * 9 + c * 3 + r];
            Mat3x3f u, vt, sg;
            svd3(a, u, vt, sg);
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 3; ++r)
                {
                    U9[p * 9 + c * 3 + r] = u(r, c);
                    Vt9[p * 9 + c * 3 + r] = vt(r, c);
                }
            S3[p * 3 + 0] = sg(0, 0);
            S3[p * 3 + 1] = sg(1, 1);
            S3[p * 3 + 2] = sg(2, 2);
        }
    }
}
