// Triangle-mesh SDF grids built on the GPU: the work of crmpm::SdfBuilder
// (src/geometry_utils/sdf_builder.cpp:84-368), which the reference runs on the host, node after
// node, with an AABB tree for the closest-point search and a clustered approximation of the
// winding number for the sign.
//
// Here every grid node is one GPU thread.  A CTA covers an 8 x 8 x 4 brick of nodes and streams
// the whole mesh through shared memory in tiles of 256 triangles; each thread evaluates, for every
// triangle, the exact winding-number term and, unless a cheap lower bound rules the triangle out,
// the exact closest point.  A second kernel takes finite differences for the gradient (and, for
// slicer meshes, writes NaN at nodes whose closest point is off the mesh).  The work is FP32 ALU
// bound: about 90 instructions per (node, triangle) pair, no DRAM traffic to speak of.
//
// Arithmetic that decides the stored values (closest point, distance, gradient) is written with
// round-to-nearest intrinsics and no fused multiply-adds, in the reference's order of operations,
// so that a node whose closest triangle is the reference's gets the reference's distance bit for
// bit.  The winding number only decides the sign and is summed exactly (all triangles, no
// clustering); the reference's approximation agrees with it wherever the number is not close to
// 0.5, that is everywhere for closed meshes.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <unordered_map>
#include <vector>

#include "mpm_engine.cuh"

namespace crb200
{
    namespace sdfb
    {
        constexpr int kTile = 256;      // triangles per shared-memory stage
        constexpr int kBrickX = 8, kBrickY = 8, kBrickZ = 4;
        constexpr float kTie = 1e-5f;   // relative width of a distance tie (slicer flags)

        struct SdfGrid
        {
            float lx, ly, lz; // lower bound
            float cell;
            int nx, ny, nz;
        };

        struct V3
        {
            float x, y, z;
        };

        // Round-to-nearest vector arithmetic without contraction into fused multiply-adds.
        __device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)}; }
        __device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
        __device__ __forceinline__ V3 operator*(V3 a, float s) { return {__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)}; }
        __device__ __forceinline__ float dotRn(V3 a, V3 b)
        {
            return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
        }
        __device__ __forceinline__ V3 vmin(V3 a, V3 b) { return {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
        __device__ __forceinline__ V3 vmax(V3 a, V3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }

        struct TriHit
        {
            float d2;   // squared distance, world units
            V3 cp;      // closest point, world coordinates
            int feature; // 0..2 vertex a, b, c; 3 edge ab; 4 edge bc; 5 edge ca; 6 interior
        };

        // Closest point of triangle (ta, tb, tc) to q by Voronoi-region tests on the dot products
        // of the edge vectors with the vertex-to-point vectors (Ericson, Real-Time Collision
        // Detection, 2005, sec. 5.1.5).  As in the reference (aabb_tree.cpp:443-471) the test runs
        // in a frame where the points' box has unit size: origin min(max(a, b), min(c, q)) (the
        // reference's expression, which is not the box minimum), scale 1 / max extent; regions are
        // tested in the reference's order, vertices a, b, c, then edges ab, bc, ca, then the face
        // (aabb_tree.cpp:336-441).
        __device__ __forceinline__ TriHit closestOnTriangle(V3 q, V3 ta, V3 tb, V3 tc)
        {
            const V3 org = vmin(vmax(ta, tb), vmin(tc, q));
            const V3 top = vmax(vmax(ta, tb), vmax(tc, q));
            const V3 ext = top - org;
            const float span = fmaxf(1e-12f, fmaxf(ext.x, fmaxf(ext.y, ext.z)));
            const float unit = __fdiv_rn(1.f, span);
            const V3 p = (q - org) * unit, a = (ta - org) * unit, b = (tb - org) * unit, c = (tc - org) * unit;
            const V3 ab = b - a, ac = c - a;
            const V3 ap = p - a, bp = p - b, cq = p - c;
            const float d1 = dotRn(ab, ap), d2 = dotRn(ac, ap);
            const float d3 = dotRn(ab, bp), d4 = dotRn(ac, bp);
            const float d5 = dotRn(ab, cq), d6 = dotRn(ac, cq);
            V3 r;
            int f;
            if (d1 <= 0.f && d2 <= 0.f)
            {
                r = a;
                f = 0;
            }
            else if (d3 >= 0.f && d3 >= d4)
            {
                r = b;
                f = 1;
            }
            else if (d6 >= 0.f && d6 >= d5)
            {
                r = c;
                f = 2;
            }
            else
            {
                const float vc = __fsub_rn(__fmul_rn(d1, d4), __fmul_rn(d3, d2));
                const float va = __fsub_rn(__fmul_rn(d3, d6), __fmul_rn(d5, d4));
                const float vb = __fsub_rn(__fmul_rn(d5, d2), __fmul_rn(d1, d6));
                if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f)
                {
                    r = a + ab * __fdiv_rn(d1, __fsub_rn(d1, d3));
                    f = 3;
                }
                else if (va <= 0.f && d4 >= d3 && d5 >= d6)
                {
                    const float num = __fsub_rn(d4, d3);
                    r = b + (c - b) * __fdiv_rn(num, __fadd_rn(num, __fsub_rn(d5, d6)));
                    f = 4;
                }
                else if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f)
                {
                    r = a + ac * __fdiv_rn(d2, __fsub_rn(d2, d6));
                    f = 5;
                }
                else
                {
                    const float inv = __fdiv_rn(1.f, __fadd_rn(__fadd_rn(va, vb), vc));
                    r = (a + ab * __fmul_rn(vb, inv)) + ac * __fmul_rn(vc, inv);
                    f = 6;
                }
            }
            const V3 e = p - r;
            TriHit h;
            h.d2 = __fmul_rn(__fmul_rn(dotRn(e, e), span), span);
            h.cp = r * span + org;
            h.feature = f;
            return h;
        }

        // One pass over the mesh per node: closest point and winding number (plain meshes) or
        // closest point and the off-mesh flag (slicer meshes).  tris holds three float4 per triangle:
        // (a, bound), (b, boundary bits), (c, 0), where bound >= the largest distance from a point
        // of the triangle to its nearest vertex and the boundary bits mark, for slicer meshes,
        // boundary vertices a, b, c (bits 0-2) and boundary edges ab, bc, ca (bits 3-5).
        template <bool Mod>
        __global__ void __launch_bounds__(kBrickX *kBrickY *kBrickZ)
            k_sdfNodes(SdfGrid g, const float4 *__restrict__ tris, int numTris, float *__restrict__ dist,
                       unsigned char *__restrict__ onMesh, float4 spine)
        {
            __shared__ float4 sT[3 * kTile];
            const int t = threadIdx.x;
            const int x = blockIdx.x * kBrickX + (t & 7);
            const int y = blockIdx.y * kBrickY + ((t >> 3) & 7);
            const int z = blockIdx.z * kBrickZ + (t >> 6);
            const bool live = x < g.nx && y < g.ny && z < g.nz;
            // queryPoint = lowerBound + (x, y, z) * cellSize (sdf_builder.cpp:117)
            const V3 q = {__fadd_rn(g.lx, __fmul_rn((float)x, g.cell)), __fadd_rn(g.ly, __fmul_rn((float)y, g.cell)),
                          __fadd_rn(g.lz, __fmul_rn((float)z, g.cell))};
            float best = INFINITY;
            V3 cp = q;
            bool off = false;
            float wind = 0.f;
            for (int base = 0; base < numTris; base += kTile)
            {
                const int cnt = min(kTile, numTris - base);
                __syncthreads();
                for (int k = t; k < 3 * cnt; k += blockDim.x)
                    sT[k] = tris[3 * (size_t)base + k];
                __syncthreads();
                for (int j = 0; j < cnt; ++j)
                {
                    const float4 A = sT[3 * j], B = sT[3 * j + 1], Cc = sT[3 * j + 2];
                    const float ax = A.x - q.x, ay = A.y - q.y, az = A.z - q.z;
                    const float bx = B.x - q.x, by = B.y - q.y, bz = B.z - q.z;
                    const float cx = Cc.x - q.x, cy = Cc.y - q.y, cz = Cc.z - q.z;
                    const float la = sqrtf(ax * ax + ay * ay + az * az);
                    const float lb = sqrtf(bx * bx + by * by + bz * bz);
                    const float lc = sqrtf(cx * cx + cy * cy + cz * cz);
                    if (!Mod)
                    {
                        // solid angle of the triangle seen from q (Van Oosterom and Strackee, 1983):
                        // the reference's exact winding term (winding_number.h:93-109) without
                        // its 1/(2 pi), applied once at the end
                        const float det = ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
                        const float den = la * lb * lc + (ax * bx + ay * by + az * bz) * lc +
                                          (bx * cx + by * cy + bz * cz) * la + (cx * ax + cy * ay + cz * az) * lb;
                        wind += atan2f(det, den);
                    }
                    // every point of the triangle lies within A.w of a vertex
                    const float lower = fminf(la, fminf(lb, lc)) - A.w;
                    if (lower > 0.f && lower * lower > best * 1.001f)
                        continue;
                    const TriHit h = closestOnTriangle(q, {A.x, A.y, A.z}, {B.x, B.y, B.z}, {Cc.x, Cc.y, Cc.z});
                    if (!Mod)
                    {
                        if (h.d2 < best)
                        {
                            best = h.d2;
                            cp = h.cp;
                        }
                    }
                    else
                    {
                        const unsigned bits = __float_as_uint(B.w);
                        const bool out = h.feature < 6 && ((bits >> h.feature) & 1u);
                        if (h.d2 < best * (1.f - kTie))
                            off = out;
                        else if (h.d2 <= best * (1.f + kTie))
                            off = off || out;
                        if (h.d2 < best)
                        {
                            best = h.d2;
                            cp = h.cp;
                        }
                    }
                }
            }
            if (!live)
                return;
            const size_t idx = ((size_t)z * g.ny + y) * g.nx + x;
            const V3 e = cp - q;
            const float d = __fsqrt_rn(dotRn(e, e)); // (closestPoint - queryPoint).norm()
            if (!Mod)
            {
                // inside where the winding number exceeds 0.5 (sdf_builder.cpp:147-153)
                dist[idx] = wind * 0.15915494309189535f > 0.5f ? -d : d;
            }
            else
            {
                dist[idx] = d;
                bool on = !off;
                if (!isnan(spine.x))
                {
                    // spine area: the positive side of the plane counts as on the mesh
                    // (sdf_builder.cpp:217-226)
                    V3 n = {spine.x, spine.y, spine.z};
                    const float s2 = dotRn(n, n);
                    n = s2 > 0.f ? n * __fdiv_rn(1.f, __fsqrt_rn(s2)) : V3{0.f, 0.f, 0.f};
                    if (__fadd_rn(dotRn(q, n), spine.w) > 0.f)
                        on = true;
                }
                onMesh[idx] = on ? 1 : 0;
            }
        }

        // Finite-difference gradient (sdf_builder.cpp:231-340): central inside, one-sided on the
        // faces of the grid, scaled by 1 / cellSize and normalised on request; slicer nodes off the
        // mesh become NaN (postProcessModSdfGradient, sdf_builder.cpp:342-367).
        template <bool Mod>
        __global__ void __launch_bounds__(256)
            k_sdfGradient(SdfGrid g, const float *__restrict__ dist, const unsigned char *__restrict__ onMesh,
                          float4 *__restrict__ out, int normalize)
        {
            const size_t n = (size_t)g.nx * g.ny * g.nz;
            const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
            if (idx >= n)
                return;
            if (Mod && !onMesh[idx])
            {
                const float nan = __int_as_float(0x7fc00000);
                out[idx] = make_float4(nan, nan, nan, nan);
                return;
            }
            const int x = (int)(idx % g.nx);
            const int y = (int)((idx / g.nx) % g.ny);
            const int z = (int)(idx / ((size_t)g.nx * g.ny));
            const float inv = __fdiv_rn(1.f, g.cell);
            const size_t sy = g.nx, sz = (size_t)g.nx * g.ny;
            auto diff = [&](int i, int ni, size_t s) {
                if (i > 0 && i < ni - 1)
                    return __fmul_rn(__fmul_rn(__fsub_rn(dist[idx + s], dist[idx - s]), 0.5f), inv);
                if (i == 0)
                    return __fmul_rn(__fsub_rn(dist[idx + s], dist[idx]), inv);
                return __fmul_rn(__fsub_rn(dist[idx], dist[idx - s]), inv);
            };
            V3 gr = {diff(x, g.nx, 1), diff(y, g.ny, sy), diff(z, g.nz, sz)};
            if (normalize)
            {
                const float s2 = dotRn(gr, gr);
                if (s2 > 0.f)
                    gr = gr * __fdiv_rn(1.f, __fsqrt_rn(s2));
            }
            out[idx] = make_float4(gr.x, gr.y, gr.z, dist[idx]);
        }

        int invalid(const char *msg)
        {
            setLastError(msg);
            return CRB200_ERR_INVALID_ARGUMENT;
        }

        int checkMesh(const CrB200TriangleMesh *m, const char *who)
        {
            if (!m || !m->points || !m->triangles)
                return invalid((std::string(who) + ": null mesh array").c_str());
            if (m->numPoints <= 0 || m->numTriangles <= 0)
                return invalid((std::string(who) + ": the mesh needs points and triangles").c_str());
            const long long np = m->numPoints;
            for (long long k = 0; k < 3LL * m->numTriangles; ++k)
                if ((long long)m->triangles[k] >= np)
                    return invalid((std::string(who) + ": triangle index out of range").c_str());
            return CRB200_OK;
        }

        // SdfBuilder::precomputeSdfDesc (sdf_builder.cpp:84-103) with the tree's root box of
        // buildTree (winding_number.h:145-156): per-triangle boxes that start at the origin, hold
        // the three vertices and are enlarged by 1e-4; their union enlarged by `fatten`.
        int precomputeDesc(CrB200SdfDesc *d, const CrB200TriangleMesh *m)
        {
            if (!d)
                return invalid("CrB200SdfPrecomputeDesc: null desc");
            if (int rc = checkMesh(m, "CrB200SdfPrecomputeDesc"))
                return rc;
            if (!(d->cellSize > 0.f) || !std::isfinite(d->fatten))
                return invalid("CrB200SdfPrecomputeDesc: cellSize must be positive and fatten finite");
            float lo[3] = {0.f, 0.f, 0.f}, hi[3] = {0.f, 0.f, 0.f};
            for (long long k = 0; k < 3LL * m->numTriangles; ++k)
            {
                const float *p = m->points + 3 * (size_t)m->triangles[k];
                for (int a = 0; a < 3; ++a)
                {
                    lo[a] = std::fmin(lo[a], p[a]);
                    hi[a] = std::fmax(hi[a], p[a]);
                }
            }
            for (int a = 0; a < 3; ++a)
            {
                // x - e is monotone in x, so the union of the enlarged boxes is the enlarged union
                float l = lo[a] - 1e-4f, h = hi[a] + 1e-4f;
                l = l - d->fatten;
                h = h + d->fatten;
                d->lowerBound[a] = l;
                d->boundingSize[a] = h - l;
                const float cells = d->boundingSize[a] / d->cellSize + 1.0f;
                if (!(cells < 2147483647.f))
                    return invalid("CrB200SdfPrecomputeDesc: grid too large");
                d->sdfDimension[a] = (int)cells;
            }
            return CRB200_OK;
        }

        int build(const CrB200SdfDesc *d, const CrB200TriangleMesh *m, CrB200Float4 *out, bool mod, int normalize,
                  cudaStream_t st)
        {
            const char *who = mod ? "CrB200SdfComputeMod" : "CrB200SdfCompute";
            if (!d || !out)
                return invalid((std::string(who) + ": null argument").c_str());
            if (int rc = checkMesh(m, who))
                return rc;
            if (!(d->cellSize > 0.f))
                return invalid((std::string(who) + ": cellSize must be positive").c_str());
            const long long nx = d->sdfDimension[0], ny = d->sdfDimension[1], nz = d->sdfDimension[2];
            if (nx < 2 || ny < 2 || nz < 2)
                return invalid((std::string(who) + ": every grid axis needs at least 2 nodes").c_str());
            const long long nodes = nx * ny * nz;
            if (nodes >= (1LL << 31) || (nz + kBrickZ - 1) / kBrickZ > 65535 || (ny + kBrickY - 1) / kBrickY > 65535)
            {
                setLastError(std::string(who) + ": grid too large");
                return CRB200_ERR_CAPACITY;
            }
            const int nt = m->numTriangles;
            // triangle records; boundary bits from the edge -> triangle count of the reference's
            // buildEdgeTriangleMap / buildEdgeVerticesList (sdf_builder.cpp:44-82)
            std::vector<float4> rec(3 * (size_t)nt);
            std::unordered_map<uint64_t, int> edgeUse;
            auto key = [](unsigned a, unsigned b) {
                return a < b ? ((uint64_t)a << 32) | b : ((uint64_t)b << 32) | a;
            };
            if (mod)
            {
                edgeUse.reserve(3 * (size_t)nt);
                for (int i = 0; i < nt; ++i)
                    for (int k = 0; k < 3; ++k)
                        ++edgeUse[key(m->triangles[3 * i + k], m->triangles[3 * i + (k + 1) % 3])];
            }
            std::vector<unsigned char> boundaryVertex;
            if (mod)
            {
                boundaryVertex.assign((size_t)m->numPoints, 0);
                for (const auto &kv : edgeUse)
                    if (kv.second < 2)
                    {
                        boundaryVertex[kv.first >> 32] = 1;
                        boundaryVertex[kv.first & 0xffffffffu] = 1;
                    }
            }
            for (int i = 0; i < nt; ++i)
            {
                const unsigned *tv = m->triangles + 3 * (size_t)i;
                const float *P[3] = {m->points + 3 * (size_t)tv[0], m->points + 3 * (size_t)tv[1],
                                     m->points + 3 * (size_t)tv[2]};
                double longest = 0.0;
                for (int k = 0; k < 3; ++k)
                {
                    const float *u = P[k], *v = P[(k + 1) % 3];
                    const double l = std::sqrt((double)(u[0] - v[0]) * (u[0] - v[0]) + (double)(u[1] - v[1]) * (u[1] - v[1]) +
                                               (double)(u[2] - v[2]) * (u[2] - v[2]));
                    longest = l > longest ? l : longest;
                }
                // no point of a triangle is farther than longest / sqrt(3) from its nearest vertex
                const float bound = (float)(longest * 0.5773502691896258 * 1.0001 + 1e-7);
                unsigned bits = 0;
                if (mod)
                {
                    for (int k = 0; k < 3; ++k)
                        bits |= (unsigned)boundaryVertex[tv[k]] << k;
                    if (edgeUse[key(tv[0], tv[1])] < 2)
                        bits |= 1u << 3;
                    if (edgeUse[key(tv[1], tv[2])] < 2)
                        bits |= 1u << 4;
                    if (edgeUse[key(tv[0], tv[2])] < 2)
                        bits |= 1u << 5;
                }
                float bitsF;
                std::memcpy(&bitsF, &bits, 4);
                rec[3 * (size_t)i + 0] = make_float4(P[0][0], P[0][1], P[0][2], bound);
                rec[3 * (size_t)i + 1] = make_float4(P[1][0], P[1][1], P[1][2], bitsF);
                rec[3 * (size_t)i + 2] = make_float4(P[2][0], P[2][1], P[2][2], 0.f);
            }

            float4 *dTris = nullptr;
            float *dDist = nullptr;
            unsigned char *dOn = nullptr;
            cudaError_t e = cudaMallocAsync(&dTris, rec.size() * sizeof(float4), st);
            if (e == cudaSuccess)
                e = cudaMallocAsync(&dDist, (size_t)nodes * sizeof(float), st);
            if (e == cudaSuccess && mod)
                e = cudaMallocAsync(&dOn, (size_t)nodes, st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(dTris, rec.data(), rec.size() * sizeof(float4), cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess)
            {
                SdfGrid g{d->lowerBound[0], d->lowerBound[1], d->lowerBound[2], d->cellSize, (int)nx, (int)ny, (int)nz};
                const float4 spine = make_float4(d->slicerSpineArea.x, d->slicerSpineArea.y, d->slicerSpineArea.z,
                                                 d->slicerSpineArea.w);
                const dim3 grid((unsigned)((nx + kBrickX - 1) / kBrickX), (unsigned)((ny + kBrickY - 1) / kBrickY),
                                (unsigned)((nz + kBrickZ - 1) / kBrickZ));
                const unsigned gb = (unsigned)((nodes + 255) / 256);
                float4 *o = reinterpret_cast<float4 *>(out);
                if (mod)
                {
                    k_sdfNodes<true><<<grid, kBrickX * kBrickY * kBrickZ, 0, st>>>(g, dTris, nt, dDist, dOn, spine);
                    k_sdfGradient<true><<<gb, 256, 0, st>>>(g, dDist, dOn, o, 1);
                }
                else
                {
                    k_sdfNodes<false><<<grid, kBrickX * kBrickY * kBrickZ, 0, st>>>(g, dTris, nt, dDist, nullptr, spine);
                    k_sdfGradient<false><<<gb, 256, 0, st>>>(g, dDist, nullptr, o, normalize);
                }
                e = cudaGetLastError();
                noteLaunches(2);
            }
            // stream-ordered frees run after the kernels
            if (dTris)
                cudaFreeAsync(dTris, st);
            if (dDist)
                cudaFreeAsync(dDist, st);
            if (dOn)
                cudaFreeAsync(dOn, st);
            if (e != cudaSuccess)
                return cudaFail(e, who);
            return CRB200_OK;
        }
    } // namespace sdfb
} // namespace crb200

extern "C"
{
    CRB200_API int CrB200SdfPrecomputeDesc(CrB200SdfDesc *desc, const CrB200TriangleMesh *mesh)
    {
        return crb200::sdfb::precomputeDesc(desc, mesh);
    }

    CRB200_API int CrB200SdfCompute(const CrB200SdfDesc *desc, const CrB200TriangleMesh *mesh,
                                    CrB200Float4 *gradientSignedDistance, int normalizeGradient, void *stream)
    {
        return crb200::sdfb::build(desc, mesh, gradientSignedDistance, false, normalizeGradient,
                                   static_cast<cudaStream_t>(stream));
    }

    CRB200_API int CrB200SdfComputeMod(const CrB200SdfDesc *desc, const CrB200TriangleMesh *mesh,
                                       CrB200Float4 *gradientSignedDistance, void *stream)
    {
        return crb200::sdfb::build(desc, mesh, gradientSignedDistance, true, 1, static_cast<cudaStream_t>(stream));
    }
}
