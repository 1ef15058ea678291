// ORACLE / TEST INFRASTRUCTURE ONLY: drives the reference's own CPU SDF builder
// (src/geometry_utils/sdf_builder.cpp: SdfBuilder::precomputeSdfDesc, computeSdf, computeModSdf,
// computeSdfGradient, postProcessModSdfGradient; AABB tree and approximate winding number from
// aabb_tree.cpp and winding_number.cpp), compiled from the reference's sources by oracle/Makefile
// (`make ref`).  It pins the CPU restatement (oracle/sdf_oracle.cpp), makes the golden grids under
// tests/golden/, and is the CPU baseline of the SDF benchmark.
#include <vector>

#include "sdf_builder.h"

using namespace crmpm;

namespace
{
    void fillMesh(const float *pts, int np, const unsigned *tris, int nt, std::vector<Vec3f3> &P,
                  std::vector<unsigned> &T, TriangleMesh &m)
    {
        P.resize(np);
        for (int i = 0; i < np; ++i)
            P[i] = Vec3f3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
        T.assign(tris, tris + 3 * nt);
        m.points = P.data();
        m.triangles = T.data();
        m.numPoints = np;
        m.numTriangles = nt;
    }
} // namespace

extern "C"
{
    // Grid of the SDF the reference builds for a mesh: dims[3], lower bound[3].
    int ref_sdf_desc(const float *pts, int np, const unsigned *tris, int nt, float cell, float fatten, int *dims,
                     float *lower)
    {
        std::vector<Vec3f3> P;
        std::vector<unsigned> T;
        TriangleMesh m;
        fillMesh(pts, np, tris, nt, P, T, m);
        SdfDesc d;
        d.cellSize = cell;
        d.fatten = fatten;
        SdfBuilder::precomputeSdfDesc(d, m);
        for (int k = 0; k < 3; ++k)
        {
            dims[k] = d.sdfDimension[k];
            lower[k] = d.lowerBound[k];
        }
        delete d.tree;
        delete d.clusters;
        return 0;
    }

    // The reference's SDF grid (gradient xyz, signed distance w per node, x fastest).
    int ref_sdf_build(const float *pts, int np, const unsigned *tris, int nt, float cell, float fatten, int normalize,
                      float *out)
    {
        std::vector<Vec3f3> P;
        std::vector<unsigned> T;
        TriangleMesh m;
        fillMesh(pts, np, tris, nt, P, T, m);
        SdfDesc d;
        d.cellSize = cell;
        d.fatten = fatten;
        SdfBuilder::precomputeSdfDesc(d, m);
        float4 *g = reinterpret_cast<float4 *>(out);
        SdfBuilder::computeSdf(d, m, g);
        SdfBuilder::computeSdfGradient(d, g, normalize != 0);
        delete d.tree;
        delete d.clusters;
        return 0;
    }

    // The reference's slicer SDF grid (computeModSdf + computeSdfGradient +
    // postProcessModSdfGradient, the sequence of simulation_factory_impl.cpp:669-684); spine[4] is
    // SdfDesc::slicerSpineArea.
    int ref_sdf_build_mod(const float *pts, int np, const unsigned *tris, int nt, float cell, float fatten,
                          const float *spine, float *out)
    {
        std::vector<Vec3f3> P;
        std::vector<unsigned> T;
        TriangleMesh m;
        fillMesh(pts, np, tris, nt, P, T, m);
        SdfDesc d;
        d.cellSize = cell;
        d.fatten = fatten;
        d.slicerSpineArea = make_float4(spine[0], spine[1], spine[2], spine[3]);
        SdfBuilder::precomputeSdfDesc(d, m);
        float4 *g = reinterpret_cast<float4 *>(out);
        Array<bool> onMesh;
        SdfBuilder::computeModSdf(d, m, g, onMesh);
        SdfBuilder::computeSdfGradient(d, g);
        SdfBuilder::postProcessModSdfGradient(d, g, onMesh);
        delete d.tree;
        delete d.clusters;
        return 0;
    }
}
