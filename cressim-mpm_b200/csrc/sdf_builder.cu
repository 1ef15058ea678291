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

#include <algorithm>
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
        constexpr int kLeaf = 8;        // triangles per leaf of the tree
        constexpr float kBeta = 2.f;    // far-field distance of a tree node, in node radii
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

        // Approximate length for bounds and the winding sum (MUFU reciprocal square root).
        __device__ __forceinline__ float fastLen(float l2) { return l2 > 0.f ? l2 * rsqrtf(l2) : 0.f; }

        // Squared distance from q to the box [lo, hi].
        __device__ __forceinline__ float boxDist2(V3 q, float4 lo, float4 hi)
        {
            const float ex = fmaxf(fmaxf(lo.x - q.x, q.x - hi.x), 0.f);
            const float ey = fmaxf(fmaxf(lo.y - q.y, q.y - hi.y), 0.f);
            const float ez = fmaxf(fmaxf(lo.z - q.z, q.z - hi.z), 0.f);
            return ex * ex + ey * ey + ez * ez;
        }

        // Implicit tree over the triangles: leaves of kLeaf triangles contiguous in Morton order of
        // their centroids, padded to a power of two P of leaves, heap-numbered (root 1, children 2n
        // and 2n + 1, leaf i at P + i).  kNodeF4 float4 per heap node: (box min, radius about the
        // centroid), (box max, triangle count: -1 inner node, 0 empty), (area-weighted centroid,
        // boundary-triangle flag), (sum of area-weighted normals, slab max), (unit mean normal n,
        // slab min): every point p of the subtree's triangles has slab min <= n . p <= slab max.
        struct TreeView
        {
            const float4 *nodes;
            const float4 *tris; // three float4 per triangle, leaf by leaf: (a, bound), (b, boundary bits),
                                // (c, original index)
            int leaves;         // P
        };

        constexpr int kNodeF4 = 5;

        // Lower bound of the squared distance from q to the triangles under a tree node: the larger
        // of the distances to its box and to its normal slab.
        __device__ __forceinline__ float nodeLower2(V3 q, const float4 *__restrict__ nd, int n, float4 lo, float4 hi)
        {
            const float4 sl = __ldg(&nd[kNodeF4 * n + 4]);
            const float smax = __ldg(&nd[kNodeF4 * n + 3]).w;
            const float s = sl.x * q.x + sl.y * q.y + sl.z * q.z;
            const float e = fmaxf(fmaxf(sl.w - s, s - smax), 0.f);
            return fmaxf(boxDist2(q, lo, hi), e * e);
        }

        // Next heap node after skipping the subtree of n (stackless depth-first order); 0 = done.
        __device__ __forceinline__ int skipSubtree(int n)
        {
            while (n & 1)
                n >>= 1;
            return n ? n + 1 : 0;
        }

        // Closest point of one triangle record against the running best; ties go to the lowest
        // original index, so the result does not depend on the visiting order.
        __device__ __forceinline__ void closestUpdate(V3 q, float4 A, float4 B, float4 Cc, float &best, int &bestId, V3 &cp)
        {
            const TriHit h = closestOnTriangle(q, {A.x, A.y, A.z}, {B.x, B.y, B.z}, {Cc.x, Cc.y, Cc.z});
            const int id = __float_as_int(Cc.w);
            if (h.d2 < best || (h.d2 == best && id < bestId))
            {
                best = h.d2;
                bestId = id;
                cp = h.cp;
            }
        }

        // Closest point and winding number (plain meshes) or closest point and the off-mesh flag
        // (slicer meshes) of one node per thread, by a walk over the implicit tree.
        //
        // Closest point: a greedy descent to the nearer child gives a first bound; the walk then
        // opens a node only when its box is no farther than the best distance so far, and tests a
        // triangle only when its nearest vertex, less the triangle's bound, is.  Winding number: a
        // node whose centroid is more than kBeta radii away contributes its dipole term and is not
        // opened for the winding number; leaves nearer than that contribute the exact solid angle of
        // each triangle.  This is the first-order far field of Barill et al., "Fast winding numbers
        // for soups and clouds" (SIGGRAPH 2018), which the reference applies on its AABB tree with
        // the same beta = 2 (sdf_builder.cpp:150, winding_number.cpp:147-170).
        template <bool Mod>
        __global__ void __launch_bounds__(kBrickX *kBrickY *kBrickZ, 4)
            k_sdfNodes(SdfGrid g, TreeView tv, float *__restrict__ dist, unsigned char *__restrict__ onMesh, float4 spine)
        {
            const int t = threadIdx.x;
            const int x = blockIdx.x * kBrickX + (t & 7);
            const int y = blockIdx.y * kBrickY + ((t >> 3) & 7);
            const int z = blockIdx.z * kBrickZ + (t >> 6);
            const bool inGrid = x < g.nx && y < g.ny && z < g.nz;
            // the walk is shared by the warp's nodes (a 8 x 4 patch): a tree node is opened when
            // any of them needs it, and each lane applies its own tests inside
            const unsigned warpMask = __ballot_sync(0xffffffffu, inGrid);
            if (!inGrid)
                return;
            // queryPoint = lowerBound + (x, y, z) * cellSize (sdf_builder.cpp:117)
            const V3 q = {__fadd_rn(g.lx, __fmul_rn((float)x, g.cell)), __fadd_rn(g.ly, __fmul_rn((float)y, g.cell)),
                          __fadd_rn(g.lz, __fmul_rn((float)z, g.cell))};
            const float4 *__restrict__ nd = tv.nodes;
            float best = INFINITY;
            int bestId = 0x7fffffff;
            V3 cp = q;

            // The walk goes down the nearer child first (nearer for the warp's first node), so that
            // the best distance tightens early: depth d, heap node n, and bit d of `second` set
            // while the walk is in the child it entered second.
            const int lead = __ffs(warpMask) - 1;
            float wind = 0.f;
            int wRoot = 0; // subtree whose winding number is already counted by its dipole
            int n = 1, depth = 0;
            unsigned second = 0;
            while (true)
            {
                bool open = false, leaf = false;
                bool needC = false, nearW = false;
                if (wRoot)
                {
                    const int sh = __clz(wRoot) - __clz(n);
                    if (sh < 0 || (n >> sh) != wRoot)
                        wRoot = 0;
                }
                const float4 lo = __ldg(&nd[kNodeF4 * n]), hi = __ldg(&nd[kNodeF4 * n + 1]);
                const int cnt = __float_as_int(hi.w);
                if (cnt != 0)
                {
                    needC = nodeLower2(q, nd, n, lo, hi) <= best * 1.001f;
                    if (!Mod && !wRoot)
                    {
                        const float4 cen = __ldg(&nd[kNodeF4 * n + 2]);
                        const float dx = cen.x - q.x, dy = cen.y - q.y, dz = cen.z - q.z;
                        const float d2 = dx * dx + dy * dy + dz * dz;
                        const float reach = kBeta * lo.w;
                        nearW = d2 <= reach * reach;
                        if (!nearW)
                        {
                            const float4 an = __ldg(&nd[kNodeF4 * n + 3]);
                            const float il = rsqrtf(d2);
                            wind += 0.5f * (an.x * dx + an.y * dy + an.z * dz) * (il * il * il);
                            wRoot = n; // the walk may still open this subtree for other needs
                        }
                    }
                    open = __any_sync(warpMask, needC || nearW);
                    leaf = cnt > 0;
                }
                if (open && !leaf)
                {
                    const int l = 2 * n;
                    const float4 hl = __ldg(&nd[kNodeF4 * l + 1]), hr = __ldg(&nd[kNodeF4 * (l + 1) + 1]);
                    const float dl = __float_as_int(hl.w) ? nodeLower2(q, nd, l, __ldg(&nd[kNodeF4 * l]), hl) : INFINITY;
                    const float dr =
                        __float_as_int(hr.w) ? nodeLower2(q, nd, l + 1, __ldg(&nd[kNodeF4 * (l + 1)]), hr) : INFINITY;
                    const bool rightFirst = __shfl_sync(warpMask, dr < dl, lead);
                    ++depth;
                    second &= ~(1u << depth);
                    n = rightFirst ? l + 1 : l;
                    continue;
                }
                if (open)
                {
                    const float4 *tr = tv.tris + 3 * (size_t)(n - tv.leaves) * kLeaf;
                    for (int j = 0; j < cnt; ++j)
                    {
                        if (!needC && !nearW)
                            continue;
                        const float4 A = __ldg(&tr[3 * j]), B = __ldg(&tr[3 * j + 1]), Cc = __ldg(&tr[3 * j + 2]);
                        const float ax = A.x - q.x, ay = A.y - q.y, az = A.z - q.z;
                        const float bx = B.x - q.x, by = B.y - q.y, bz = B.z - q.z;
                        const float cx = Cc.x - q.x, cy = Cc.y - q.y, cz = Cc.z - q.z;
                        const float la = fastLen(ax * ax + ay * ay + az * az);
                        const float lb = fastLen(bx * bx + by * by + bz * bz);
                        const float lc = fastLen(cx * cx + cy * cy + cz * cz);
                        if (!Mod && nearW)
                        {
                            // solid angle of the triangle seen from q (Van Oosterom and Strackee, 1983):
                            // the reference's exact winding term (winding_number.h:93-109) without
                            // its 1/(2 pi), applied once at the end
                            const float det = ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
                            const float den = la * lb * lc + (ax * bx + ay * by + az * bz) * lc +
                                              (bx * cx + by * cy + bz * cz) * la + (cx * ax + cy * ay + cz * az) * lb;
                            wind += atan2f(det, den);
                        }
                        if (!needC)
                            continue;
                        // every point of the triangle lies within A.w of a vertex, and none is nearer to q
                        // than the triangle's plane; the plane bound is used for triangles whose smallest
                        // angle at a has a sine above 0.01, where the float normal's direction is good to
                        // 1e-5, and is lowered by that error times the vertex distance
                        float lower = fminf(la, fminf(lb, lc)) * 0.9999f - A.w;
                        {
                            const float e1x = B.x - A.x, e1y = B.y - A.y, e1z = B.z - A.z;
                            const float e2x = Cc.x - A.x, e2y = Cc.y - A.y, e2z = Cc.z - A.z;
                            const float nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
                            const float n2 = nx * nx + ny * ny + nz * nz;
                            const float s12 = (e1x * e1x + e1y * e1y + e1z * e1z) * (e2x * e2x + e2y * e2y + e2z * e2z);
                            if (n2 > 1e-4f * s12)
                            {
                                const float plane = fabsf(nx * ax + ny * ay + nz * az) * rsqrtf(n2);
                                lower = fmaxf(lower, plane * 0.9999f - 1e-5f * la);
                            }
                        }
                        if (lower > 0.f && lower * lower > best * 1.001f)
                            continue;
                        closestUpdate(q, A, B, Cc, best, bestId, cp);
                    }
                }
                // next: climb out of the subtrees entered second, then cross to the sibling
                while (depth > 0 && ((second >> depth) & 1u))
                {
                    second &= ~(1u << depth);
                    --depth;
                    n >>= 1;
                }
                if (depth == 0)
                    break;
                second |= 1u << depth;
                n ^= 1;
            }

            const size_t idx = ((size_t)z * g.ny + y) * g.nx + x;
            const V3 e = cp - q;
            const float d = __fsqrt_rn(dotRn(e, e)); // (closestPoint - queryPoint).norm()
            if (!Mod)
            {
                // inside where the winding number exceeds 0.5 (sdf_builder.cpp:147-153)
                dist[idx] = wind * 0.15915494309189535f > 0.5f ? -d : d;
                return;
            }
            // off the mesh when any triangle within kTie of the closest distance has its closest
            // point on a boundary vertex or boundary edge (aabb_tree.cpp:523-625)
            const float tie = best * (1.f + kTie);
            bool off = false;
            n = 1;
            while (n)
            {
                const float4 lo = __ldg(&nd[kNodeF4 * n]), hi = __ldg(&nd[kNodeF4 * n + 1]);
                const int cnt = __float_as_int(hi.w);
                // .w of the third float4 flags subtrees holding a triangle with boundary bits
                const bool open = cnt != 0 && __ldg(&nd[kNodeF4 * n + 2]).w != 0.f &&
                                  nodeLower2(q, nd, n, lo, hi) <= tie * 1.001f;
                if (!__any_sync(warpMask, open && !off))
                {
                    n = skipSubtree(n);
                    continue;
                }
                if (cnt < 0)
                {
                    n = 2 * n;
                    continue;
                }
                const float4 *tr = tv.tris + 3 * (size_t)(n - tv.leaves) * kLeaf;
                for (int j = 0; j < cnt; ++j)
                {
                    const float4 A = __ldg(&tr[3 * j]), B = __ldg(&tr[3 * j + 1]), Cc = __ldg(&tr[3 * j + 2]);
                    const unsigned bits = __float_as_uint(B.w);
                    if (!bits || !open || off)
                        continue;
                    const TriHit h = closestOnTriangle(q, {A.x, A.y, A.z}, {B.x, B.y, B.z}, {Cc.x, Cc.y, Cc.z});
                    if (h.d2 <= tie && h.feature < 6 && ((bits >> h.feature) & 1u))
                        off = true;
                }
                n = skipSubtree(n);
            }
            dist[idx] = d;
            bool on = !off;
            if (!isnan(spine.x))
            {
                // spine area: the positive side of the plane counts as on the mesh
                // (sdf_builder.cpp:217-226)
                V3 sn = {spine.x, spine.y, spine.z};
                const float s2 = dotRn(sn, sn);
                sn = s2 > 0.f ? sn * __fdiv_rn(1.f, __fsqrt_rn(s2)) : V3{0.f, 0.f, 0.f};
                if (__fadd_rn(dotRn(q, sn), spine.w) > 0.f)
                    on = true;
            }
            onMesh[idx] = on ? 1 : 0;
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

        // Events around the kernels of the most recent build on this host thread.
        struct KernelClock
        {
            cudaEvent_t begin = nullptr, mid = nullptr, end = nullptr;
            bool recorded = false;
            ~KernelClock()
            {
                for (cudaEvent_t e : {begin, mid, end})
                    if (e)
                        cudaEventDestroy(e);
            }
        };
        thread_local KernelClock tClock;

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
            // boundary bits from the edge -> triangle count of the reference's buildEdgeTriangleMap /
            // buildEdgeVerticesList (sdf_builder.cpp:44-82)
            std::unordered_map<uint64_t, int> edgeUse;
            auto key = [](unsigned a, unsigned b) {
                return a < b ? ((uint64_t)a << 32) | b : ((uint64_t)b << 32) | a;
            };
            std::vector<unsigned char> boundaryVertex;
            if (mod)
            {
                edgeUse.reserve(3 * (size_t)nt);
                for (int i = 0; i < nt; ++i)
                    for (int k = 0; k < 3; ++k)
                        ++edgeUse[key(m->triangles[3 * i + k], m->triangles[3 * i + (k + 1) % 3])];
                boundaryVertex.assign((size_t)m->numPoints, 0);
                for (const auto &kv : edgeUse)
                    if (kv.second < 2)
                    {
                        boundaryVertex[kv.first >> 32] = 1;
                        boundaryVertex[kv.first & 0xffffffffu] = 1;
                    }
            }
            auto vert = [&](int i, int k) { return m->points + 3 * (size_t)m->triangles[3 * (size_t)i + k]; };

            // triangle centroids
            std::vector<double> cen(3 * (size_t)nt);
            for (int i = 0; i < nt; ++i)
                for (int a = 0; a < 3; ++a)
                    cen[3 * (size_t)i + a] = ((double)vert(i, 0)[a] + vert(i, 1)[a] + vert(i, 2)[a]) / 3.0;
            // leaves of kLeaf triangles; the implicit tree above them (see TreeView)
            const int nLeaves = (nt + kLeaf - 1) / kLeaf;
            int P = 1;
            while (P < nLeaves)
                P <<= 1;
            // Top-down split of the centroids: a node's triangles are ordered along the longest axis
            // of their centroids' box and its left child takes as many as its subtree holds (half the
            // node's slots), so filled leaves form a prefix and every subtree is spatially compact.
            std::vector<uint64_t> order(nt);
            {
                std::vector<int> ord(nt);
                for (int i = 0; i < nt; ++i)
                    ord[i] = i;
                struct Span
                {
                    int b, e;
                    long long cap;
                };
                std::vector<Span> todo{{0, nt, (long long)P * kLeaf}};
                while (!todo.empty())
                {
                    const Span sp = todo.back();
                    todo.pop_back();
                    if (sp.cap <= kLeaf || sp.e - sp.b <= 1)
                        continue;
                    const long long half = sp.cap / 2;
                    const int m = sp.b + (int)std::min<long long>(sp.e - sp.b, half);
                    if (m < sp.e)
                    {
                        double blo[3] = {INFINITY, INFINITY, INFINITY}, bhi[3] = {-INFINITY, -INFINITY, -INFINITY};
                        for (int k = sp.b; k < sp.e; ++k)
                            for (int a = 0; a < 3; ++a)
                            {
                                blo[a] = std::fmin(blo[a], cen[3 * (size_t)ord[k] + a]);
                                bhi[a] = std::fmax(bhi[a], cen[3 * (size_t)ord[k] + a]);
                            }
                        int axis = 0;
                        for (int a = 1; a < 3; ++a)
                            if (bhi[a] - blo[a] > bhi[axis] - blo[axis])
                                axis = a;
                        std::nth_element(ord.begin() + sp.b, ord.begin() + m, ord.begin() + sp.e, [&](int u, int v) {
                            const double cu = cen[3 * (size_t)u + axis], cv = cen[3 * (size_t)v + axis];
                            return cu < cv || (cu == cv && u < v);
                        });
                    }
                    todo.push_back({sp.b, m, half});
                    todo.push_back({m, sp.e, half});
                }
                for (int k = 0; k < nt; ++k)
                    order[k] = (uint64_t)ord[k];
            }
            std::vector<float4> rec(3 * (size_t)P * kLeaf, make_float4(0.f, 0.f, 0.f, 0.f));
            std::vector<float4> tree(kNodeF4 * (size_t)(2 * P));
            std::vector<double> area(2 * (size_t)P, 0.0), wc(3 * 2 * (size_t)P, 0.0), an(3 * 2 * (size_t)P, 0.0);
            std::vector<unsigned char> anyBits(2 * (size_t)P, 0);
            const float4 emptyLo = make_float4(INFINITY, INFINITY, INFINITY, 0.f);
            auto intBits = [](int v) {
                float f;
                std::memcpy(&f, &v, 4);
                return f;
            };
            auto asInt = [](float f) {
                int v;
                std::memcpy(&v, &f, 4);
                return v;
            };
            for (int lf = 0; lf < P; ++lf)
            {
                const size_t h = (size_t)P + lf;
                const int first = lf * kLeaf, cnt = lf < nLeaves ? std::min(kLeaf, nt - first) : 0;
                float blo[3] = {INFINITY, INFINITY, INFINITY}, bhi[3] = {-INFINITY, -INFINITY, -INFINITY};
                for (int j = 0; j < cnt; ++j)
                {
                    const int i = (int)(order[first + j] & 0xffffffffu);
                    const unsigned *tv = m->triangles + 3 * (size_t)i;
                    const float *Pv[3] = {vert(i, 0), vert(i, 1), vert(i, 2)};
                    double longest = 0.0;
                    for (int k = 0; k < 3; ++k)
                    {
                        const float *u = Pv[k], *v = Pv[(k + 1) % 3];
                        const double l = std::sqrt((double)(u[0] - v[0]) * (u[0] - v[0]) + (double)(u[1] - v[1]) * (u[1] - v[1]) +
                                                   (double)(u[2] - v[2]) * (u[2] - v[2]));
                        longest = l > longest ? l : longest;
                        for (int a = 0; a < 3; ++a)
                        {
                            blo[a] = std::fmin(blo[a], u[a]);
                            bhi[a] = std::fmax(bhi[a], u[a]);
                        }
                    }
                    // no point of a triangle is farther than longest / sqrt(3) from its nearest vertex
                    const float bound = (float)(longest * 0.5773502691896258 * 1.0001 + 1e-7);
                    unsigned bits = 0;
                    if (mod)
                    {
                        for (int k = 0; k < 3; ++k)
                            bits |= (unsigned)boundaryVertex[tv[k]] << k;
                        bits |= (unsigned)(edgeUse[key(tv[0], tv[1])] < 2) << 3;
                        bits |= (unsigned)(edgeUse[key(tv[1], tv[2])] < 2) << 4;
                        bits |= (unsigned)(edgeUse[key(tv[0], tv[2])] < 2) << 5;
                    }
                    anyBits[h] |= bits ? 1 : 0;
                    float bitsF;
                    std::memcpy(&bitsF, &bits, 4);
                    const size_t r = 3 * ((size_t)first + j);
                    rec[r + 0] = make_float4(Pv[0][0], Pv[0][1], Pv[0][2], bound);
                    rec[r + 1] = make_float4(Pv[1][0], Pv[1][1], Pv[1][2], bitsF);
                    rec[r + 2] = make_float4(Pv[2][0], Pv[2][1], Pv[2][2], intBits(i));
                    // dipole data as the reference's precomputeClusterInformation / approximateCluster
                    // (winding_number.cpp:47-78, 121-142): area-weighted centroid, summed half cross
                    // products, radius = farthest vertex from the centroid
                    double e1[3], e2[3];
                    for (int a = 0; a < 3; ++a)
                    {
                        e1[a] = (double)Pv[1][a] - Pv[0][a];
                        e2[a] = (double)Pv[2][a] - Pv[0][a];
                    }
                    const double hx = 0.5 * (e1[1] * e2[2] - e1[2] * e2[1]), hy = 0.5 * (e1[2] * e2[0] - e1[0] * e2[2]),
                                 hz = 0.5 * (e1[0] * e2[1] - e1[1] * e2[0]);
                    const double ar = std::sqrt(hx * hx + hy * hy + hz * hz);
                    an[3 * h] += hx, an[3 * h + 1] += hy, an[3 * h + 2] += hz;
                    area[h] += ar;
                    for (int a = 0; a < 3; ++a)
                        wc[3 * h + a] += ar * cen[3 * (size_t)i + a];
                }
                tree[kNodeF4 * h + 0] = cnt ? make_float4(blo[0], blo[1], blo[2], 0.f) : emptyLo;
                tree[kNodeF4 * h + 1] = cnt ? make_float4(bhi[0], bhi[1], bhi[2], intBits(cnt))
                                       : make_float4(-INFINITY, -INFINITY, -INFINITY, intBits(0));
            }
            for (int h = P - 1; h >= 1; --h)
            {
                const size_t l = 2 * (size_t)h, r = l + 1;
                const int cl = asInt(tree[kNodeF4 * l + 1].w), cr = asInt(tree[kNodeF4 * r + 1].w);
                anyBits[h] = anyBits[l] | anyBits[r];
                area[h] = area[l] + area[r];
                for (int a = 0; a < 3; ++a)
                {
                    an[3 * h + a] = an[3 * l + a] + an[3 * r + a];
                    wc[3 * h + a] = wc[3 * l + a] + wc[3 * r + a];
                }
                const float4 ll = tree[kNodeF4 * l], lh = tree[kNodeF4 * l + 1], rl = tree[kNodeF4 * r],
                             rh = tree[kNodeF4 * r + 1];
                tree[kNodeF4 * (size_t)h + 0] = make_float4(std::fmin(ll.x, rl.x), std::fmin(ll.y, rl.y), std::fmin(ll.z, rl.z), 0.f);
                tree[kNodeF4 * (size_t)h + 1] = make_float4(std::fmax(lh.x, rh.x), std::fmax(lh.y, rh.y), std::fmax(lh.z, rh.z),
                                                       intBits(cl == 0 && cr == 0 ? 0 : -1));
            }
            // centroids, radii (farthest vertex of the subtree from its centroid), flags
            int levels = 0;
            while ((1 << levels) < P)
                ++levels;
            for (size_t h = 1; h < 2 * (size_t)P; ++h)
            {
                float4 &lo4 = tree[kNodeF4 * h];
                if (asInt(tree[kNodeF4 * h + 1].w) == 0)
                {
                    tree[kNodeF4 * h + 2] = make_float4(0.f, 0.f, 0.f, 0.f);
                    tree[kNodeF4 * h + 3] = make_float4(0.f, 0.f, 0.f, INFINITY);
                    tree[kNodeF4 * h + 4] = make_float4(0.f, 0.f, 0.f, -INFINITY);
                    continue;
                }
                const float4 hi4 = tree[kNodeF4 * h + 1];
                double c[3] = {0.5 * ((double)lo4.x + hi4.x), 0.5 * ((double)lo4.y + hi4.y), 0.5 * ((double)lo4.z + hi4.z)};
                if (area[h] > 0) // degenerate (zero-area) subtrees keep their box centre
                    for (int a = 0; a < 3; ++a)
                        c[a] = wc[3 * h + a] / area[h];
                int depth = 0;
                while ((2ull << depth) <= h)
                    ++depth;
                const int span = 1 << (levels - depth);
                const size_t firstLeaf = (h << (levels - depth)) - P;
                // unit mean normal, as the float the kernel multiplies by
                const double al = std::sqrt(an[3 * h] * an[3 * h] + an[3 * h + 1] * an[3 * h + 1] + an[3 * h + 2] * an[3 * h + 2]);
                const float un[3] = {al > 0 ? (float)(an[3 * h] / al) : 0.f, al > 0 ? (float)(an[3 * h + 1] / al) : 0.f,
                                     al > 0 ? (float)(an[3 * h + 2] / al) : 0.f};
                double r2 = 0.0, smin = INFINITY, smax = -INFINITY, reach = 0.0;
                for (size_t lf = firstLeaf; lf < firstLeaf + span && lf < (size_t)nLeaves; ++lf)
                    for (int j = 0; j < kLeaf && (int)(lf * kLeaf) + j < nt; ++j)
                        for (int k = 0; k < 3; ++k)
                        {
                            const float4 v = rec[3 * (lf * kLeaf + j) + k];
                            const double dx = v.x - c[0], dy = v.y - c[1], dz = v.z - c[2];
                            r2 = std::fmax(r2, dx * dx + dy * dy + dz * dz);
                            const double sv = (double)un[0] * v.x + (double)un[1] * v.y + (double)un[2] * v.z;
                            smin = std::fmin(smin, sv);
                            smax = std::fmax(smax, sv);
                            reach = std::fmax(reach, std::fabs(v.x) + std::fabs(v.y) + std::fabs(v.z));
                        }
                // widen the slab by the rounding of the kernel's float dot product n . q (q within the
                // grid, which is within the mesh's reach plus the fatten distance)
                const double slack = 1e-6 * (1.0 + reach + 3.0 * std::fabs((double)d->fatten));
                lo4.w = (float)(std::sqrt(r2) * 1.0001);
                tree[kNodeF4 * h + 2] = make_float4((float)c[0], (float)c[1], (float)c[2], anyBits[h] ? 1.f : 0.f);
                tree[kNodeF4 * h + 3] = make_float4((float)an[3 * h], (float)an[3 * h + 1], (float)an[3 * h + 2],
                                                    al > 0 ? std::nextafter((float)(smax + slack), INFINITY) : INFINITY);
                tree[kNodeF4 * h + 4] = make_float4(un[0], un[1], un[2],
                                                    al > 0 ? std::nextafter((float)(smin - slack), -INFINITY) : -INFINITY);
            }
            const size_t triRecords = rec.size();
            rec.insert(rec.end(), tree.begin(), tree.end()); // one upload: triangles, then the tree

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
                const TreeView tv{dTris + triRecords, dTris, P};
                if (!tClock.begin)
                {
                    cudaEventCreate(&tClock.begin);
                    cudaEventCreate(&tClock.mid);
                    cudaEventCreate(&tClock.end);
                }
                tClock.recorded = false;
                cudaEventRecord(tClock.begin, st);
                if (mod)
                {
                    k_sdfNodes<true><<<grid, kBrickX * kBrickY * kBrickZ, 0, st>>>(g, tv, dDist, dOn, spine);
                    cudaEventRecord(tClock.mid, st);
                    k_sdfGradient<true><<<gb, 256, 0, st>>>(g, dDist, dOn, o, 1);
                }
                else
                {
                    k_sdfNodes<false><<<grid, kBrickX * kBrickY * kBrickZ, 0, st>>>(g, tv, dDist, nullptr, spine);
                    cudaEventRecord(tClock.mid, st);
                    k_sdfGradient<false><<<gb, 256, 0, st>>>(g, dDist, nullptr, o, normalize);
                }
                cudaEventRecord(tClock.end, st);
                e = cudaGetLastError();
                tClock.recorded = e == cudaSuccess;
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

    CRB200_API int CrB200SdfGetLastKernelTime(float outMs[2])
    {
        using crb200::sdfb::tClock;
        if (!outMs)
            return crb200::sdfb::invalid("CrB200SdfGetLastKernelTime: null argument");
        if (!tClock.recorded)
            return crb200::sdfb::invalid("CrB200SdfGetLastKernelTime: no SDF build on this thread");
        cudaError_t e = cudaEventSynchronize(tClock.end);
        if (e == cudaSuccess)
            e = cudaEventElapsedTime(&outMs[0], tClock.begin, tClock.mid);
        if (e == cudaSuccess)
            e = cudaEventElapsedTime(&outMs[1], tClock.mid, tClock.end);
        return e == cudaSuccess ? CRB200_OK : crb200::cudaFail(e, "CrB200SdfGetLastKernelTime");
    }

    CRB200_API int CrB200SdfComputeMod(const CrB200SdfDesc *desc, const CrB200TriangleMesh *mesh,
                                       CrB200Float4 *gradientSignedDistance, void *stream)
    {
        return crb200::sdfb::build(desc, mesh, gradientSignedDistance, true, 1, static_cast<cudaStream_t>(stream));
    }
}
