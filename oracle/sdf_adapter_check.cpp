// ORACLE / TEST INFRASTRUCTURE ONLY: runs the reference-side SDF adapter
// (cressim-mpm_b200/adapter/gpu_b200_sdf_builder.h, which calls libcrmpm_b200.so on the GPU) and
// the reference's own SdfBuilder (src/geometry_utils/sdf_builder.cpp, compiled in by
// `make -C oracle ref`) on the same mesh, as SimulationFactoryImpl::createGeometry would call them.
//
//     sdf_adapter_check mesh.bin cell fatten slicer
//
// mesh.bin: int32 numPoints, int32 numTriangles, float32 points[3 * numPoints], uint32
// triangles[3 * numTriangles].  Prints the grid dimensions, the number of nodes whose distance
// differs, the largest distance difference, the nodes whose NaN (off-mesh) state differs and
// whose sign differs, and exits 0 when the descriptors agree.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "gpu_b200_sdf_builder.h"

using namespace crmpm;

int main(int argc, char **argv)
{
    if (argc < 5)
        return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f)
        return 2;
    int np = 0, nt = 0;
    if (std::fread(&np, 4, 1, f) != 1 || std::fread(&nt, 4, 1, f) != 1)
        return 2;
    std::vector<Vec3f3> P(np);
    std::vector<unsigned> T(3 * (size_t)nt);
    std::vector<float> raw(3 * (size_t)np);
    if (std::fread(raw.data(), 4, raw.size(), f) != raw.size() || std::fread(T.data(), 4, T.size(), f) != T.size())
        return 2;
    std::fclose(f);
    for (int i = 0; i < np; ++i)
        P[i] = Vec3f3(raw[3 * i], raw[3 * i + 1], raw[3 * i + 2]);
    TriangleMesh mesh;
    mesh.points = P.data();
    mesh.triangles = T.data();
    mesh.numPoints = np;
    mesh.numTriangles = nt;
    const float cell = (float)std::atof(argv[2]), fatten = (float)std::atof(argv[3]);
    const bool slicer = std::atoi(argv[4]) != 0;

    SdfDesc ref, gpu;
    ref.cellSize = gpu.cellSize = cell;
    ref.fatten = gpu.fatten = fatten;
    SdfBuilder::precomputeSdfDesc(ref, mesh);
    GpuB200SdfBuilder::precomputeSdfDesc(gpu, mesh);
    bool same = true;
    for (int a = 0; a < 3; ++a)
        same = same && ref.sdfDimension[a] == gpu.sdfDimension[a] && ref.lowerBound[a] == gpu.lowerBound[a];
    const size_t n = (size_t)ref.sdfDimension[0] * ref.sdfDimension[1] * ref.sdfDimension[2];
    std::vector<float4> a(n), b(n);
    if (slicer)
    {
        Array<bool> onMesh;
        SdfBuilder::computeModSdf(ref, mesh, a.data(), onMesh);
        SdfBuilder::computeSdfGradient(ref, a.data());
        SdfBuilder::postProcessModSdfGradient(ref, a.data(), onMesh);
        GpuB200SdfBuilder::computeModSdfWithGradient(gpu, mesh, b.data());
    }
    else
    {
        SdfBuilder::computeSdf(ref, mesh, a.data());
        SdfBuilder::computeSdfGradient(ref, a.data());
        GpuB200SdfBuilder::computeSdfWithGradient(gpu, mesh, b.data());
    }
    size_t differ = 0, nanDiffer = 0, signDiffer = 0;
    double maxDiff = 0.0;
    for (size_t i = 0; i < n; ++i)
    {
        const bool na = std::isnan(a[i].w), nb = std::isnan(b[i].w);
        if (na != nb)
        {
            ++nanDiffer;
            continue;
        }
        if (na)
            continue;
        if (a[i].w != b[i].w)
            ++differ;
        if ((a[i].w < 0.f) != (b[i].w < 0.f) && a[i].w != 0.f && b[i].w != 0.f)
            ++signDiffer;
        maxDiff = std::fmax(maxDiff, std::fabs((double)a[i].w - (double)b[i].w));
    }
    std::printf("dims %dx%dx%d nodes %zu differ %zu maxdiff %.3e nan_differ %zu sign_differ %zu desc_same %d\n",
                ref.sdfDimension[0], ref.sdfDimension[1], ref.sdfDimension[2], n, differ, maxDiff, nanDiffer,
                signDiffer, same ? 1 : 0);
    delete ref.tree;
    delete ref.clusters;
    return same ? 0 : 1;
}
