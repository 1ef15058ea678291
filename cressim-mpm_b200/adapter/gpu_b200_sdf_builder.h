// Drop-in for the SdfBuilder calls of SimulationFactoryImpl::createGeometry
// (src/engine/simulation_factory_impl.cpp:630-641 for eTriangleMesh, :669-684 for
// eTriangleMeshSlicer): the SDF grid is computed on the GPU by libcrmpm_b200.so
// (CrB200SdfPrecomputeDesc / CrB200SdfCompute / CrB200SdfComputeMod) and copied into the factory's
// host SDF array, which the factory then uploads as before.
//
// In createGeometry,
//     SdfBuilder::precomputeSdfDesc(sdfDesc, mesh);
//     ...
//     SdfBuilder::computeSdf(sdfDesc, mesh, out);
//     SdfBuilder::computeSdfGradient(sdfDesc, out);
// becomes
//     GpuB200SdfBuilder::precomputeSdfDesc(sdfDesc, mesh);
//     ...
//     GpuB200SdfBuilder::computeSdfWithGradient(sdfDesc, mesh, out);
// and the slicer's computeModSdf + computeSdfGradient + postProcessModSdfGradient becomes
// GpuB200SdfBuilder::computeModSdfWithGradient(sdfDesc, mesh, out).  The descriptor gets no AABB
// tree or winding-number clusters (tree and clusters stay null): nothing after the build reads them.
// Errors are logged the way the reference logs CUDA errors and execution continues.
#ifndef CR_GPU_B200_SDF_BUILDER_H
#define CR_GPU_B200_SDF_BUILDER_H

#include <cuda_runtime.h>

#include <cstdio>

#include "crmpm_b200.h"
#include "sdf_builder.h"

namespace crmpm
{
    class GpuB200SdfBuilder
    {
    public:
        // SdfBuilder::precomputeSdfDesc (src/geometry_utils/sdf_builder.cpp:84-103).
        static void precomputeSdfDesc(SdfDesc &d, TriangleMesh &mesh)
        {
            CrB200TriangleMesh m = toMesh(mesh);
            CrB200SdfDesc c = toDesc(d);
            check(CrB200SdfPrecomputeDesc(&c, &m));
            d.lowerBound = Vec3f(c.lowerBound[0], c.lowerBound[1], c.lowerBound[2]);
            d.boundingSize = Vec3f(c.boundingSize[0], c.boundingSize[1], c.boundingSize[2]);
            d.sdfDimension = Vec3i(c.sdfDimension[0], c.sdfDimension[1], c.sdfDimension[2]);
            d.tree = nullptr;
            d.clusters = nullptr;
        }

        // SdfBuilder::computeSdf followed by computeSdfGradient (sdf_builder.cpp:105-161, 231-340),
        // into the host array gradientDistance (dimX * dimY * dimZ float4).
        static void computeSdfWithGradient(SdfDesc &d, TriangleMesh &mesh, float4 *gradientDistance,
                                           bool normalize = true)
        {
            build(false, d, mesh, gradientDistance, normalize);
        }

        // SdfBuilder::computeModSdf, computeSdfGradient and postProcessModSdfGradient
        // (sdf_builder.cpp:163-229, 231-340, 342-367) for slicer meshes.
        static void computeModSdfWithGradient(SdfDesc &d, TriangleMesh &mesh, float4 *gradientDistance)
        {
            build(true, d, mesh, gradientDistance, true);
        }

    private:
        static CrB200TriangleMesh toMesh(const TriangleMesh &mesh)
        {
            return CrB200TriangleMesh{reinterpret_cast<const float *>(mesh.points), mesh.triangles, mesh.numPoints,
                                      mesh.numTriangles};
        }

        static CrB200SdfDesc toDesc(const SdfDesc &d)
        {
            CrB200SdfDesc c{};
            c.cellSize = d.cellSize;
            c.fatten = d.fatten;
            c.slicerSpineArea = CrB200Float4{d.slicerSpineArea.x, d.slicerSpineArea.y, d.slicerSpineArea.z,
                                             d.slicerSpineArea.w};
            for (int a = 0; a < 3; ++a)
            {
                c.lowerBound[a] = d.lowerBound[a];
                c.boundingSize[a] = d.boundingSize[a];
                c.sdfDimension[a] = d.sdfDimension[a];
            }
            return c;
        }

        static void build(bool mod, SdfDesc &d, TriangleMesh &mesh, float4 *host, bool normalize)
        {
            const size_t n = (size_t)d.sdfDimension[0] * d.sdfDimension[1] * d.sdfDimension[2];
            CrB200TriangleMesh m = toMesh(mesh);
            CrB200SdfDesc c = toDesc(d);
            CrB200Float4 *dev = nullptr;
            if (cudaMalloc(&dev, n * sizeof(CrB200Float4)) != cudaSuccess)
            {
                std::fprintf(stderr, "crmpm_b200 error: cannot allocate the SDF grid on the device\n");
                return;
            }
            const int rc = mod ? CrB200SdfComputeMod(&c, &m, dev, nullptr)
                               : CrB200SdfCompute(&c, &m, dev, normalize ? 1 : 0, nullptr);
            check(rc);
            if (rc == CRB200_OK &&
                cudaMemcpy(host, dev, n * sizeof(CrB200Float4), cudaMemcpyDeviceToHost) != cudaSuccess)
                std::fprintf(stderr, "crmpm_b200 error: SDF grid copy failed\n");
            cudaFree(dev);
        }

        static void check(int rc)
        {
            if (rc != CRB200_OK)
                std::fprintf(stderr, "crmpm_b200 error %d: %s\n", rc, CrB200GetLastError());
        }

        static_assert(sizeof(Vec3f3) == 3 * sizeof(float), "TriangleMesh points are packed float triples");
        static_assert(sizeof(float4) == sizeof(CrB200Float4), "float4 layout");
    };
} // namespace crmpm

#endif // !CR_GPU_B200_SDF_BUILDER_H
