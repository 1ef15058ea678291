// An MLS-MPM substep that allocates no memory: CrB200MlsSubstepNoAlloc.
//
// Who needs it: callers that must not (or cannot) call cudaMalloc from the thread that steps the
// simulation -- a host that has already partitioned all device memory among its own pools, a
// process that runs the step from inside a real-time control loop where an allocation's
// synchronisation and latency are not acceptable, or code that only owns the particle buffers
// it was handed.  The regular solver (CrB200SolverCreate / CrB200SolverInitialize) allocates its
// sort buffers and grids up front; this entry point instead keeps its only scratch -- the two
// node grids of the substep and the shape table -- in a file-scope device array of fixed size,
// which every GPU that loads the library holds until the process exits.
//
// Limits and sharing rules:
//   * at most kNoAllocMaxNodes grid nodes (nx * ny * nz) and kMaxShapes shapes per call;
//     larger requests are rejected with CRB200_ERR_CAPACITY before anything is launched;
//   * all calls share the one scratch array, so two calls that overlap on the GPU (different
//     streams, or different host threads) race and corrupt each other's grids: serialise them;
//   * the first call on a device looks up the array's device address (cudaGetSymbolAddress with
//     that device current); make that first call before any stream capture.  The address is kept
//     for the life of the process, so a device reset (cudaDeviceReset, or anything else that
//     destroys the primary context) after that first call is not supported: later calls would
//     use an address of the destroyed context.
// The arithmetic is the regular MLS substep (mls_mpm_algorithm.h:147-390 of the reference):
// per-particle P2G with float4 vector atomics into a dense grid, the grid update with SDF contact
// and domain boundary, and G2P; only the grid layout (dense, x fastest) and the scratch source
// differ, so results agree with CrB200SolverStep to float32 rounding.

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "mpm_engine.cuh"

namespace crb200
{
    namespace noalloc
    {
        constexpr unsigned kNoAllocMaxNodes = 1u << 18; // 262,144 nodes per grid (2 grids: 8 MiB)

        // accumulation grid [0, kNoAllocMaxNodes), velocity grid [kNoAllocMaxNodes, 2x)
        static __device__ __align__(256) float4 g_scratchGrid[2 * kNoAllocMaxNodes];
        static __device__ __align__(256) ShapeRec g_scratchShapes[kMaxShapes];
        static __device__ int g_scratchFlags; // shape flags of the current call (SF_*)

        struct Geo
        {
            float3 gmin, gmax;
            float dx, invDx;
            int nx, ny, nz;
        };

        __device__ __forceinline__ bool inside(const Geo &g, int i, int j, int k)
        {
            return i >= 0 && i < g.nx && j >= 0 && j < g.ny && k >= 0 && k < g.nz;
        }

        // baseCoord / fx (mls_mpm_algorithm.h:170-175), exactly rounded
        __device__ __forceinline__ void stencil(const Geo &g, V3 x, int b[3], float f[3], bool &finite)
        {
            const float sp[3] = {ex::mul(ex::sub(x.x, g.gmin.x), g.invDx), ex::mul(ex::sub(x.y, g.gmin.y), g.invDx),
                                 ex::mul(ex::sub(x.z, g.gmin.z), g.invDx)};
            finite = fabsf(sp[0]) < 1.0e7f && fabsf(sp[1]) < 1.0e7f && fabsf(sp[2]) < 1.0e7f;
#pragma unroll
            for (int d = 0; d < 3; ++d)
            {
                b[d] = finite ? __float2int_rz(ex::sub(sp[d], 0.5f)) : 0;
                f[d] = ex::sub(sp[d], (float)b[d]);
            }
        }

        __device__ __forceinline__ void bspline(const float f[3], float w[3][3])
        {
#pragma unroll
            for (int d = 0; d < 3; ++d)
            {
                const float a = 1.5f - f[d], b = f[d] - 1.0f, c = f[d] - 0.5f;
                w[0][d] = 0.5f * (a * a);
                w[1][d] = 0.75f - b * b;
                w[2][d] = 0.5f * (c * c);
            }
        }

        __global__ void k_clearAndGather(unsigned numNodes, float4 *__restrict__ gridA, int numShapes,
                                         const int *__restrict__ shapeIds, CrB200ShapeData sh, CrB200GeometryData ge,
                                         ShapeRec *__restrict__ table, int *__restrict__ flagsOut)
        {
            const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
            for (unsigned n = t; n < numNodes; n += gridDim.x * blockDim.x)
                gridA[n] = make_float4(0.f, 0.f, 0.f, 0.f); // the previous call's contents are stale
            if (blockIdx.x == 0)
            {
                __shared__ int flags;
                if (threadIdx.x == 0)
                    flags = 0;
                __syncthreads();
                for (int s = threadIdx.x; s < numShapes; s += blockDim.x)
                {
                    const ShapeRec r = makeShapeRec(shapeIds[s], sh, ge);
                    table[s] = r;
                    atomicOr(&flags, shapeFlagsOf(r));
                }
                __syncthreads();
                if (threadIdx.x == 0)
                    *flagsOut = flags;
            }
        }

        __global__ void __launch_bounds__(128) k_p2g(Geo g, float dt, float3 gravity, unsigned n,
                                                     const float4 *__restrict__ xm, const float4 *__restrict__ vel,
                                                     const float *__restrict__ F, const float *__restrict__ Cm,
                                                     const float *__restrict__ V0, const float4 *__restrict__ matParams,
                                                     const int *__restrict__ matType, const unsigned char *__restrict__ mask,
                                                     int numShapes, const ShapeRec *__restrict__ table,
                                                     const int *__restrict__ flags, SdfPtrs sdf, float4 *__restrict__ gridA)
        {
            __shared__ ShapeRec sh[kMaxShapes];
            const bool slicers = numShapes > 0 && (*flags & SF_SLICER);
            if (slicers)
            {
                for (int s = threadIdx.x; s < numShapes; s += blockDim.x)
                    sh[s] = table[s];
                __syncthreads();
            }
            const unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
            if (p >= n || !mask[p])
                return;
            const float4 x4 = xm[p];
            const V3 x = v3(x4);
            int b[3];
            float f[3];
            bool finite;
            stencil(g, x, b, f, finite);
            if (!finite)
                return;
            float w[3][3];
            bspline(f, w);
            M3 Fp, Cp;
#pragma unroll
            for (int e = 0; e < 9; ++e)
            {
                Fp.m[e] = F[9 * p + e];
                Cp.m[e] = Cm[9 * p + e];
            }
            const float m = x4.w;
            const float4 mp = matParams[p];
            const M3 s = kirchhoffStress(Fp, mp.x, mp.y, matType[p]);
            const float coef = -dt * 4.f * g.invDx * g.invDx * V0[p];
            M3 A;
#pragma unroll
            for (int e = 0; e < 9; ++e)
                A.m[e] = s.m[e] * coef + Cp.m[e] * m;
            const V3 mv = (v3(vel[p]) + v3(gravity) * dt) * m;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int k = 0; k < 3; ++k)
                    {
                        const int ni = b[0] + i, nj = b[1] + j, nk = b[2] + k;
                        if (!inside(g, ni, nj, nk))
                            continue;
                        const V3 d = v3(ex::mul(ex::sub((float)i, f[0]), g.dx), ex::mul(ex::sub((float)j, f[1]), g.dx),
                                        ex::mul(ex::sub((float)k, f[2]), g.dx));
                        if (slicers && differentSides(x, ex::add(x, d), sh, numShapes, sdf, nullptr))
                            continue;
                        const float wt = w[i][0] * w[j][1] * w[k][2];
                        const V3 ad = v3(A.m[0] * d.x + A.m[3] * d.y + A.m[6] * d.z, A.m[1] * d.x + A.m[4] * d.y + A.m[7] * d.z,
                                         A.m[2] * d.x + A.m[5] * d.y + A.m[8] * d.z);
                        const V3 c = (mv + ad) * wt;
                        atomicAdd(&gridA[ni + g.nx * (nj + g.ny * nk)], make_float4(c.x, c.y, c.z, wt * m));
                    }
        }

        __global__ void __launch_bounds__(256) k_update(Geo g, float dt, unsigned numNodes, int numShapes, int contactModel,
                                                        const ShapeRec *__restrict__ table, SdfPtrs sdf,
                                                        const float4 *__restrict__ gridA, float4 *__restrict__ gridV,
                                                        float4 *coupleForce, float4 *coupleTorque)
        {
            __shared__ ShapeRec sh[kMaxShapes];
            if (numShapes > 0)
            {
                for (int s = threadIdx.x; s < numShapes; s += blockDim.x)
                    sh[s] = table[s];
                __syncthreads();
            }
            const unsigned n = blockIdx.x * blockDim.x + threadIdx.x;
            if (n >= numNodes)
                return;
            const int i = n % g.nx, j = (n / g.nx) % g.ny, k = n / (g.nx * g.ny);
            const float4 a = gridA[n];
            if (a.w < 1e-4f)
            {
                gridV[n] = a; // light nodes keep momentum (mls_mpm_algorithm.h:265-266)
                return;
            }
            V3 v = v3(a.x / a.w, a.y / a.w, a.z / a.w);
            V3 pos = v3((float)i * g.dx, (float)j * g.dx, (float)k * g.dx) + v3(g.gmin) + v * dt;
            if (numShapes > 0)
                {
                    CoupleAtomic couple{coupleForce, coupleTorque};
                    rigidContact<false>(v, a.w, pos, sh, numShapes, sdf, contactModel == 1, couple);
                }
            if (i < 2 || i > g.nx - 3)
                v.x = 0.f;
            if (j < 2 || j > g.ny - 3)
                v.y = 0.f;
            if (k < 2 || k > g.nz - 3)
                v.z = 0.f;
            gridV[n] = make_float4(v.x, v.y, v.z, a.w);
        }

        __global__ void __launch_bounds__(128) k_g2p(Geo g, float dt, float3 gravity, unsigned n, float4 *__restrict__ xm,
                                                     float4 *__restrict__ vel, float *__restrict__ F, float *__restrict__ Cm,
                                                     const unsigned char *__restrict__ mask, int numShapes,
                                                     const ShapeRec *__restrict__ table, const int *__restrict__ flags,
                                                     SdfPtrs sdf, const float4 *__restrict__ gridV)
        {
            __shared__ ShapeRec sh[kMaxShapes];
            if (numShapes > 0)
            {
                for (int s = threadIdx.x; s < numShapes; s += blockDim.x)
                    sh[s] = table[s];
                __syncthreads();
            }
            const unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
            if (p >= n || !mask[p])
                return;
            const bool slicers = numShapes > 0 && (*flags & SF_SLICER);
            const float4 x4 = xm[p];
            const V3 x = v3(x4);
            int b[3];
            float f[3];
            bool finite;
            stencil(g, x, b, f, finite);
            float w[3][3];
            bspline(f, w);
            const V3 vk = v3(vel[p]) + v3(gravity) * dt; // the velocity P2G kicked
            V3 va = v3(0.f, 0.f, 0.f);
            float Ca[9];
#pragma unroll
            for (int e = 0; e < 9; ++e)
                Ca[e] = 0.f;
            if (finite)
            {
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j)
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                        {
                            const int ni = b[0] + i, nj = b[1] + j, nk = b[2] + k;
                            if (!inside(g, ni, nj, nk))
                                continue;
                            V3 nv = v3(gridV[ni + g.nx * (nj + g.ny * nk)]);
                            const V3 d = v3(ex::mul(ex::sub((float)i, f[0]), g.dx), ex::mul(ex::sub((float)j, f[1]), g.dx),
                                            ex::mul(ex::sub((float)k, f[2]), g.dx));
                            V3 nrm;
                            if (slicers && differentSides(x, ex::add(x, d), sh, numShapes, sdf, &nrm))
                                nv = vk - nrm * dot(vk, nrm) * 2.0f;
                            const V3 nw = nv * (w[i][0] * w[j][1] * w[k][2]);
                            va = va + nw;
                            // reference outerProduct(nw, d): M(r, c) = nw_c * d_r
                            Ca[0] += nw.x * d.x;
                            Ca[1] += nw.x * d.y;
                            Ca[2] += nw.x * d.z;
                            Ca[3] += nw.y * d.x;
                            Ca[4] += nw.y * d.y;
                            Ca[5] += nw.y * d.z;
                            Ca[6] += nw.z * d.x;
                            Ca[7] += nw.z * d.y;
                            Ca[8] += nw.z * d.z;
                        }
            }
            M3 Cn, Mu, Fp;
            const float s4 = 4.f * g.invDx;
#pragma unroll
            for (int e = 0; e < 9; ++e)
            {
                Cn.m[e] = Ca[e] * s4;
                Mu.m[e] = ((e % 4) == 0 ? 1.f : 0.f) + Cn.m[e] * dt;
                Fp.m[e] = F[9 * p + e];
            }
            V3 xn = x + va * dt;
            xn = v3(fminf(fmaxf(xn.x, g.gmin.x), g.gmax.x), fminf(fmaxf(xn.y, g.gmin.y), g.gmax.y),
                    fminf(fmaxf(xn.z, g.gmin.z), g.gmax.z));
            V3 vn = va;
            if (numShapes > 0)
                {
                    CoupleAtomic noCouple{nullptr, nullptr};
                    rigidContact<true>(vn, x4.w, xn, sh, numShapes, sdf, false, noCouple);
                }
            Fp = matmul(Mu, Fp);
            xm[p] = make_float4(xn.x, xn.y, xn.z, x4.w);
            vel[p] = make_float4(vn.x, vn.y, vn.z, 0.f);
#pragma unroll
            for (int e = 0; e < 9; ++e)
            {
                F[9 * p + e] = Fp.m[e];
                Cm[9 * p + e] = Cn.m[e];
            }
        }

        // Per-device addresses of the scratch arrays, looked up once per device.
        struct DevicePtrs
        {
            float4 *grid = nullptr;
            ShapeRec *shapes = nullptr;
            int *flags = nullptr;
        };
        static std::mutex g_mutex;
        static DevicePtrs g_ptrs[64];

        int devicePtrs(DevicePtrs &out)
        {
            int dev = 0;
            cudaError_t e = cudaGetDevice(&dev);
            if (e != cudaSuccess)
                return cudaFail(e, "CrB200MlsSubstepNoAlloc: cudaGetDevice");
            if (dev < 0 || dev >= 64)
            {
                setLastError("CrB200MlsSubstepNoAlloc: device ordinal above 63");
                return CRB200_ERR_UNSUPPORTED;
            }
            std::lock_guard<std::mutex> lock(g_mutex);
            DevicePtrs &d = g_ptrs[dev];
            if (!d.grid)
            {
                void *pg = nullptr, *ps = nullptr, *pf = nullptr;
                e = cudaGetSymbolAddress(&pg, g_scratchGrid);
                if (e != cudaSuccess)
                    return cudaFail(e, "CrB200MlsSubstepNoAlloc: cudaGetSymbolAddress(grid scratch)");
                e = cudaGetSymbolAddress(&ps, g_scratchShapes);
                if (e != cudaSuccess)
                    return cudaFail(e, "CrB200MlsSubstepNoAlloc: cudaGetSymbolAddress(shape scratch)");
                e = cudaGetSymbolAddress(&pf, g_scratchFlags);
                if (e != cudaSuccess)
                    return cudaFail(e, "CrB200MlsSubstepNoAlloc: cudaGetSymbolAddress(flags scratch)");
                d.grid = static_cast<float4 *>(pg);
                d.shapes = static_cast<ShapeRec *>(ps);
                d.flags = static_cast<int *>(pf);
            }
            out = d;
            return CRB200_OK;
        }

    } // namespace noalloc
} // namespace crb200

using namespace crb200;

extern "C" CRB200_API int CrB200MlsSubstepNoAlloc(const CrB200NoAllocStep *step, void *stream)
{
    if (!step)
    {
        setLastError("CrB200MlsSubstepNoAlloc: null step description");
        return CRB200_ERR_INVALID_ARGUMENT;
    }
    const CrB200NoAllocStep &s = *step;
    if (!(s.cellSize > 0.f) || !(s.dt > 0.f))
    {
        setLastError("CrB200MlsSubstepNoAlloc: cellSize and dt must be positive");
        return CRB200_ERR_INVALID_ARGUMENT;
    }
    noalloc::Geo g;
    int dims[3];
    for (int d = 0; d < 3; ++d)
    {
        if (!(s.gridMax[d] > s.gridMin[d]))
        {
            setLastError("CrB200MlsSubstepNoAlloc: empty grid bounds");
            return CRB200_ERR_INVALID_ARGUMENT;
        }
        // int((max - min) / dx + 1) in float, as the reference solvers compute it
        volatile float size = s.gridMax[d] - s.gridMin[d];
        volatile float q = size / s.cellSize;
        dims[d] = (int)(q + 1.0f);
    }
    g.gmin = make_float3(s.gridMin[0], s.gridMin[1], s.gridMin[2]);
    g.gmax = make_float3(s.gridMax[0], s.gridMax[1], s.gridMax[2]);
    g.dx = s.cellSize;
    g.invDx = 1 / s.cellSize;
    g.nx = dims[0];
    g.ny = dims[1];
    g.nz = dims[2];
    const double nodes = (double)g.nx * (double)g.ny * (double)g.nz;
    if (g.nx < 5 || g.ny < 5 || g.nz < 5)
    {
        setLastError("CrB200MlsSubstepNoAlloc: the grid needs at least 5 nodes per dimension");
        return CRB200_ERR_INVALID_ARGUMENT;
    }
    if (nodes > (double)noalloc::kNoAllocMaxNodes)
    {
        setLastError("CrB200MlsSubstepNoAlloc: grid has more than 262144 nodes, the fixed scratch limit");
        return CRB200_ERR_CAPACITY;
    }
    if (s.numShapes < 0 || s.numShapes > kMaxShapes)
    {
        setLastError("CrB200MlsSubstepNoAlloc: at most 64 shapes");
        return CRB200_ERR_CAPACITY;
    }
    if (s.numParticles > 0 && (!s.positionMass || !s.velocity || !s.F || !s.C || !s.V0 || !s.matParams || !s.matType ||
                               !s.activeMask))
    {
        setLastError("CrB200MlsSubstepNoAlloc: null particle buffer");
        return CRB200_ERR_INVALID_ARGUMENT;
    }
    if (s.numShapes > 0 &&
        (!s.shapeIds || !s.shapes.type || !s.shapes.geometryIdx || !s.shapes.position || !s.shapes.rotation ||
         !s.shapes.invScale || !s.shapes.linearVelocity || !s.shapes.angularVelocity || !s.shapes.params0 ||
         !s.shapes.force || !s.shapes.torque || !s.geometries.type || !s.geometries.params0))
    {
        setLastError("CrB200MlsSubstepNoAlloc: shapes enabled but shape ids or a shape / geometry array the substep "
                     "reads or writes (type, geometryIdx, position, rotation, invScale, linearVelocity, "
                     "angularVelocity, params0, force, torque; geometry type, params0) is null");
        return CRB200_ERR_INVALID_ARGUMENT;
    }
    // the kernels read these arrays as float4: an address off a 16-byte boundary would be a
    // misaligned access on the GPU, so it is refused here (as CrB200SolverBindParticleData does)
    {
        const void *vec4[] = {s.positionMass, s.velocity, s.matParams};
        for (const void *q : vec4)
            if (s.numParticles > 0 && (reinterpret_cast<uintptr_t>(q) & 15u) != 0)
            {
                setLastError("CrB200MlsSubstepNoAlloc: positionMass, velocity and matParams must be 16-byte aligned");
                return CRB200_ERR_INVALID_ARGUMENT;
            }
        const void *shape4[] = {s.shapes.position, s.shapes.rotation, s.shapes.invScale, s.shapes.linearVelocity,
                                s.shapes.angularVelocity, s.shapes.params0, s.shapes.force, s.shapes.torque,
                                s.shapes.comInvMass, s.shapes.inertiaInv0, s.shapes.inertiaInv1, s.geometries.params0};
        for (const void *q : shape4)
            if (s.numShapes > 0 && (reinterpret_cast<uintptr_t>(q) & 15u) != 0)
            {
                setLastError("CrB200MlsSubstepNoAlloc: shape and geometry float4 arrays must be 16-byte aligned");
                return CRB200_ERR_INVALID_ARGUMENT;
            }
    }
    noalloc::DevicePtrs ptrs;
    int rc = noalloc::devicePtrs(ptrs);
    if (rc != CRB200_OK)
        return rc;
    int *flags = ptrs.flags;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const unsigned numNodes = (unsigned)nodes;
    float4 *gridA = ptrs.grid, *gridV = ptrs.grid + noalloc::kNoAllocMaxNodes;
    const SdfPtrs sdf{reinterpret_cast<const int4 *>(s.sdf.dimension), reinterpret_cast<const float4 *>(s.sdf.lowerBoundCellSize),
                      reinterpret_cast<const float4 *>(s.sdf.gradientSignedDistance)};
    const float3 grav = make_float3(s.gravity[0], s.gravity[1], s.gravity[2]);
    noalloc::k_clearAndGather<<<148 * 4, 256, 0, st>>>(numNodes, gridA, s.numShapes, s.shapeIds, s.shapes, s.geometries,
                                                       ptrs.shapes, flags);
    const unsigned pg = (s.numParticles + 127) / 128;
    if (pg)
        noalloc::k_p2g<<<pg, 128, 0, st>>>(g, s.dt, grav, s.numParticles, reinterpret_cast<const float4 *>(s.positionMass),
                                           reinterpret_cast<const float4 *>(s.velocity), s.F, s.C, s.V0,
                                           reinterpret_cast<const float4 *>(s.matParams), s.matType, s.activeMask,
                                           s.numShapes, ptrs.shapes, flags, sdf, gridA);
    noalloc::k_update<<<(numNodes + 255) / 256, 256, 0, st>>>(g, s.dt, numNodes, s.numShapes, s.contactModel, ptrs.shapes,
                                                              sdf, gridA, gridV, reinterpret_cast<float4 *>(s.shapes.force),
                                                              reinterpret_cast<float4 *>(s.shapes.torque));
    if (pg)
        noalloc::k_g2p<<<pg, 128, 0, st>>>(g, s.dt, grav, s.numParticles, reinterpret_cast<float4 *>(s.positionMass),
                                           reinterpret_cast<float4 *>(s.velocity), s.F, s.C, s.activeMask, s.numShapes,
                                           ptrs.shapes, flags, sdf, gridV);
    noteLaunches(pg ? 4 : 2);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return cudaFail(e, "CrB200MlsSubstepNoAlloc: kernel launch");
    return CRB200_OK;
}
