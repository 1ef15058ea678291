// ORACLE / TEST INFRASTRUCTURE ONLY: CPU restatement of the triangle-mesh SDF build of
// crmpm::SdfBuilder (src/geometry_utils/sdf_builder.cpp:84-368) used to check the GPU builder
// (cressim-mpm_b200/csrc/sdf_builder.cu).  Brute force over all triangles per node, in the
// reference's single-precision arithmetic (built with -ffp-contract=off):
//   - grid: precomputeSdfDesc (sdf_builder.cpp:84-103) over the tree root box of buildTree
//     (include/geometry_utils/winding_number.h:145-156), whose triangle boxes start at the origin;
//   - distance: closest point by distancePointTriangleSquared2UnitBox (aabb_tree.cpp:336-471), the
//     smallest squared distance over all triangles, then |closest point - query|
//     (sdf_builder.cpp:142-143);
//   - sign: winding number > 0.5 (sdf_builder.cpp:147-153), here the exact sum over all
//     triangles of the term of evaluateExact (winding_number.h:93-109);
//   - slicer meshes: unsigned distance; off the mesh where the closest feature of any triangle
//     within a relative 1e-5 of the smallest squared distance is a boundary vertex or boundary edge
//     (aabb_tree.cpp:523-625, 724-760), on the mesh on the positive side of the spine plane
//     (sdf_builder.cpp:217-226); NaN nodes off the mesh after the gradient (sdf_builder.cpp:342-367);
//   - gradient: computeSdfGradient (sdf_builder.cpp:231-340).
// The reference itself (oracle/_ref/libref_sdf.so, built by `make ref`) pins this restatement.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <utility>
#include <vector>

namespace
{
    struct V
    {
        float x, y, z;
    };
    V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
    V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
    V operator*(V a, float s) { return {a.x * s, a.y * s, a.z * s}; }
    float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
    V vmin(V a, V b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
    V vmax(V a, V b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }

    // Region of the closest point: 0..2 vertex a, b, c; 3 ab; 4 bc; 5 ca; 6 face.
    float closest(V q, V ta, V tb, V tc, V &out, int &feature)
    {
        const V org = vmin(vmax(ta, tb), vmin(tc, q)); // the reference's frame origin, as written
        const V top = vmax(vmax(ta, tb), vmax(tc, q));
        const V ext = top - org;
        const float span = std::fmax(1e-12f, std::fmax(ext.x, std::fmax(ext.y, ext.z)));
        const float unit = 1.f / span;
        const V p = (q - org) * unit, a = (ta - org) * unit, b = (tb - org) * unit, c = (tc - org) * unit;
        const V ab = b - a, ac = c - a;
        const float d1 = dot(ab, p - a), d2 = dot(ac, p - a);
        const float d3 = dot(ab, p - b), d4 = dot(ac, p - b);
        const float d5 = dot(ab, p - c), d6 = dot(ac, p - c);
        V r;
        if (d1 <= 0.f && d2 <= 0.f)
            r = a, feature = 0;
        else if (d3 >= 0.f && d3 >= d4)
            r = b, feature = 1;
        else if (d6 >= 0.f && d6 >= d5)
            r = c, feature = 2;
        else
        {
            const float vc = d1 * d4 - d3 * d2, va = d3 * d6 - d5 * d4, vb = d5 * d2 - d1 * d6;
            if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f)
                r = a + ab * (d1 / (d1 - d3)), feature = 3;
            else if (va <= 0.f && d4 >= d3 && d5 >= d6)
                r = b + (c - b) * ((d4 - d3) / ((d4 - d3) + (d5 - d6))), feature = 4;
            else if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f)
                r = a + ac * (d2 / (d2 - d6)), feature = 5;
            else
            {
                const float inv = 1.f / (va + vb + vc);
                r = (a + ab * (vb * inv)) + ac * (vc * inv);
                feature = 6;
            }
        }
        const V e = p - r;
        out = r * span + org;
        return dot(e, e) * span * span;
    }

    uint64_t edgeKey(unsigned a, unsigned b) { return a < b ? ((uint64_t)a << 32) | b : ((uint64_t)b << 32) | a; }
} // namespace

extern "C"
{
    // dims[3], lower[3], size[3] of the grid the reference lays over the mesh.
    int oracle_sdf_desc(const float *pts, const unsigned *tris, int nt, float cell, float fatten, int *dims,
                        float *lower, float *size)
    {
        float lo[3] = {0.f, 0.f, 0.f}, hi[3] = {0.f, 0.f, 0.f};
        for (long k = 0; k < 3L * nt; ++k)
            for (int a = 0; a < 3; ++a)
            {
                lo[a] = std::fmin(lo[a], pts[3 * tris[k] + a]);
                hi[a] = std::fmax(hi[a], pts[3 * tris[k] + a]);
            }
        for (int a = 0; a < 3; ++a)
        {
            const float l = (lo[a] - 1e-4f) - fatten, h = (hi[a] + 1e-4f) + fatten;
            lower[a] = l;
            size[a] = h - l;
            dims[a] = (int)(size[a] / cell + 1.0f);
        }
        return 0;
    }

    // Grid of float4 (gradient xyz, distance w), x fastest.  mod != 0: the slicer variant with
    // spine plane spine[4] (spine[0] NaN = none).
    int oracle_sdf_build(const float *pts, int np, const unsigned *tris, int nt, const int *dims, const float *lower,
                         float cell, int mod, const float *spine, int normalize, float *out)
    {
        const int nx = dims[0], ny = dims[1], nz = dims[2];
        const long n = (long)nx * ny * nz;
        std::vector<float> w(n);
        std::vector<char> on(n, 1);
        std::vector<unsigned> bits(nt, 0);
        if (mod)
        {
            std::map<uint64_t, int> use;
            for (int i = 0; i < nt; ++i)
                for (int k = 0; k < 3; ++k)
                    ++use[edgeKey(tris[3 * i + k], tris[3 * i + (k + 1) % 3])];
            std::vector<char> bv(np, 0);
            for (auto &kv : use)
                if (kv.second < 2)
                    bv[kv.first >> 32] = bv[kv.first & 0xffffffffu] = 1;
            for (int i = 0; i < nt; ++i)
            {
                const unsigned *t = tris + 3 * i;
                for (int k = 0; k < 3; ++k)
                    bits[i] |= (unsigned)bv[t[k]] << k;
                bits[i] |= (unsigned)(use[edgeKey(t[0], t[1])] < 2) << 3;
                bits[i] |= (unsigned)(use[edgeKey(t[1], t[2])] < 2) << 4;
                bits[i] |= (unsigned)(use[edgeKey(t[0], t[2])] < 2) << 5;
            }
        }
        auto P = [&](unsigned i) { return V{pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]}; };
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x)
                {
                    const long idx = ((long)z * ny + y) * nx + x;
                    const V q = {lower[0] + (float)x * cell, lower[1] + (float)y * cell, lower[2] + (float)z * cell};
                    float best = INFINITY;
                    V cp = q;
                    bool off = false;
                    double wind = 0.0;
                    for (int i = 0; i < nt; ++i)
                    {
                        const V a = P(tris[3 * i]), b = P(tris[3 * i + 1]), c = P(tris[3 * i + 2]);
                        if (!mod)
                        {
                            const V A = a - q, B = b - q, Cc = c - q;
                            const double la = std::sqrt((double)dot(A, A)), lb = std::sqrt((double)dot(B, B)),
                                         lc = std::sqrt((double)dot(Cc, Cc));
                            const double det = (double)A.x * ((double)B.y * Cc.z - (double)B.z * Cc.y) -
                                               (double)A.y * ((double)B.x * Cc.z - (double)B.z * Cc.x) +
                                               (double)A.z * ((double)B.x * Cc.y - (double)B.y * Cc.x);
                            const double den = la * lb * lc + (double)dot(A, B) * lc + (double)dot(B, Cc) * la +
                                               (double)dot(Cc, A) * lb;
                            wind += std::atan2(det, den);
                        }
                        V h;
                        int f;
                        const float d2 = closest(q, a, b, c, h, f);
                        if (d2 < best)
                            best = d2, cp = h;
                    }
                    if (mod)
                    {
                        // every triangle within a relative 1e-5 of the closest squared distance
                        const float tie = best * (1.f + 1e-5f);
                        for (int i = 0; i < nt && !off; ++i)
                        {
                            V h;
                            int f;
                            const float d2 = closest(q, P(tris[3 * i]), P(tris[3 * i + 1]), P(tris[3 * i + 2]), h, f);
                            off = d2 <= tie && f < 6 && ((bits[i] >> f) & 1u);
                        }
                    }
                    const V e = cp - q;
                    const float d = std::sqrt(dot(e, e));
                    if (!mod)
                        w[idx] = wind / (2.0 * M_PI) > 0.5 ? -d : d;
                    else
                    {
                        w[idx] = d;
                        on[idx] = !off;
                        if (!std::isnan(spine[0]))
                        {
                            V nn = {spine[0], spine[1], spine[2]};
                            const float s2 = dot(nn, nn);
                            nn = s2 > 0.f ? nn * (1.f / std::sqrt(s2)) : V{0.f, 0.f, 0.f};
                            if (dot(q, nn) + spine[3] > 0.f)
                                on[idx] = 1;
                        }
                    }
                }
        const float inv = 1.f / cell;
        auto D = [&](int i, int ni, long idx, long s) {
            if (i > 0 && i < ni - 1)
                return (w[idx + s] - w[idx - s]) * 0.5f * inv;
            if (i == 0)
                return (w[idx + s] - w[idx]) * inv;
            return (w[idx] - w[idx - s]) * inv;
        };
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x)
                {
                    const long idx = ((long)z * ny + y) * nx + x;
                    float *o = out + 4 * idx;
                    if (mod && !on[idx])
                    {
                        o[0] = o[1] = o[2] = o[3] = NAN;
                        continue;
                    }
                    V g = {D(x, nx, idx, 1), D(y, ny, idx, nx), D(z, nz, idx, (long)nx * ny)};
                    if (normalize)
                    {
                        const float s2 = dot(g, g);
                        if (s2 > 0.f)
                            g = g * (1.f / std::sqrt(s2));
                    }
                    o[0] = g.x, o[1] = g.y, o[2] = g.z, o[3] = w[idx];
                }
        return 0;
    }
}
