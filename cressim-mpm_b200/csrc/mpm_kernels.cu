// sm_100a kernels of the B200 MPM substep engine and the host Solver that launches them.
//
// One substep (MLS-MPM; the reference's GpuMlsMpmSolver::step, gpu_mls_mpm_solver.cu:102-109):
//   1. gatherShapes   scene shapes -> compact table (shapes may change between substeps); with the
//                     slicer cut masks on a side stream beside the sort chain
//   2. bin            per particle: cell key (block-major), rank among its cell's particles, cell
//                     and block counts (warp-aggregated atomics); done by the previous G2P when
//                     it can be
//   3. scan           block offsets, active-block list, touched-block list (3 kernels), then the
//                     absolute start of every cell of the active blocks
//   4. scatter        particle ids into their cells' slots (cells contiguous in key order; arrival
//                     order inside a cell; the canonical order is produced on request)
//   5. p2g            one CTA per active block: particles -> shared-memory 6x6x6 node tile ->
//                     one float4 vector atomic per touched node into the accumulation grid
//   6. gridUpdate     touched blocks only: momentum -> velocity, SDF contact/friction, domain BC,
//                     and the accumulation grid is zeroed as it is consumed
//   7. g2p            particle order: 27-node gather, APIC matrix, advection, push-out, F update
// PB-MPM runs 6-8 `iterations` times per step plus an integration kernel (gpu_pb_mpm_solver.cu:
// 102-113); standard MPM carries a node force tile (gpu_standard_mpm_solver.cu:177-184).

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <string>
#include <type_traits>

#include "mpm_engine.cuh"

namespace crb200
{
    constexpr unsigned kInvalidKey = 0xFFFFFFFFu;
    constexpr int kTileEdge = 6;
    constexpr int kTileNodes = kTileEdge * kTileEdge * kTileEdge;
    constexpr int kScanTile = 256; // blocks per scan tile
    constexpr int kScanThreads = 256;

    // ---------------------------------------------------------------------------------------
    // Addressing helpers
    __device__ __forceinline__ unsigned nodeAddr(const GridGeom &g, int i, int j, int k)
    {
        const unsigned b = g.blockBase + (unsigned)((i >> 2) + g.nb.x * ((j >> 2) + g.nb.y * (k >> 2)));
        return b * 64u + (unsigned)((i & 3) + 4 * ((j & 3) + 4 * (k & 3)));
    }
    __device__ __forceinline__ bool inGrid(const GridGeom &g, int i, int j, int k)
    {
        return i >= 0 && i < g.n.x && j >= 0 && j < g.n.y && k >= 0 && k < g.n.z;
    }

    struct Stencil
    {
        int b[3];
        V3 fx;
        bool finite;
    };

    // baseCoord / fx of mls_mpm_algorithm.h:170-175, exactly rounded.
    __device__ __forceinline__ Stencil stencilOf(const GridGeom &g, V3 x)
    {
        Stencil s;
        const float sp[3] = {ex::mul(ex::sub(x.x, g.gmin.x), g.invDx), ex::mul(ex::sub(x.y, g.gmin.y), g.invDx),
                             ex::mul(ex::sub(x.z, g.gmin.z), g.invDx)};
        s.finite = fabsf(sp[0]) < 1.0e7f && fabsf(sp[1]) < 1.0e7f && fabsf(sp[2]) < 1.0e7f;
        float f[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            s.b[d] = s.finite ? __float2int_rz(ex::sub(sp[d], 0.5f)) : 0;
            f[d] = ex::sub(sp[d], (float)s.b[d]);
        }
        s.fx = v3(f[0], f[1], f[2]);
        return s;
    }

    // Quadratic B-spline weights (shape_functions.h:44-57) and gradients (:62-75).
    __device__ __forceinline__ void weights(V3 fx, float w[3][3])
    {
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            const float f = comp(fx, d);
            const float a = 1.5f - f, b = f - 1.0f, c = f - 0.5f;
            w[0][d] = 0.5f * (a * a);
            w[1][d] = 0.75f - b * b;
            w[2][d] = 0.5f * (c * c);
        }
    }
    __device__ __forceinline__ void weightGrads(V3 fx, float dw[3][3])
    {
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            const float f = comp(fx, d);
            dw[0][d] = f - 1.5f;
            dw[1][d] = 2.0f * (1.0f - f);
            dw[2][d] = f - 0.5f;
        }
    }

    // Sort key: block-major cell index of the clamped base cell; outliers (a base outside the
    // grid) are binned at the nearest cell, where the P2G tile still covers every in-grid node
    // of their stencil.
    __device__ __forceinline__ unsigned cellKey(const GridGeom &g, const Stencil &s, bool *outOfDomain)
    {
        int c[3];
        const int hi[3] = {g.n.x - 2, g.n.y - 2, g.n.z - 2};
        bool ood = false;
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            c[d] = min(max(s.b[d], 0), max(hi[d], 0));
            ood |= (c[d] != s.b[d]);
        }
        *outOfDomain = ood;
        const unsigned blk = g.blockBase + (unsigned)((c[0] >> 2) + g.nb.x * ((c[1] >> 2) + g.nb.y * (c[2] >> 2)));
        return blk * 64u + (unsigned)((c[0] & 3) + 4 * ((c[1] & 3) + 4 * (c[2] & 3)));
    }

    // The region of grid block (bx, by, bz) that its shape masks cover: nodes 4b .. 4b+3 and
    // particles whose base cell lies in the block, each moved by up to two cells (cell units
    // 4b - 2 .. 4b + 6 per axis).
    struct BlockRegion
    {
        V3 lo, hi;
        __device__ __forceinline__ bool contains(V3 p) const
        {
            return p.x >= lo.x && p.x <= hi.x && p.y >= lo.y && p.y <= hi.y && p.z >= lo.z && p.z <= hi.z;
        }
    };
    __device__ __forceinline__ BlockRegion blockRegion(const GridGeom &g, int bx, int by, int bz)
    {
        BlockRegion r;
        r.lo = v3(g.gmin.x + (float)(4 * bx - 2) * g.dx, g.gmin.y + (float)(4 * by - 2) * g.dx,
                  g.gmin.z + (float)(4 * bz - 2) * g.dx);
        r.hi = v3(g.gmin.x + (float)(4 * bx + 6) * g.dx, g.gmin.y + (float)(4 * by + 6) * g.dx,
                  g.gmin.z + (float)(4 * bz + 6) * g.dx);
        return r;
    }
    // bounding ball of a region, its radius padded against rounding
    __device__ __forceinline__ void regionBall(const BlockRegion &r, V3 &c, float &R)
    {
        c = (r.lo + r.hi) * 0.5f;
        const V3 h = (r.hi - r.lo) * 0.5f;
        R = sqrtf(sq(h)) * 1.001f + 1e-6f;
    }
    // Block of a particle's (clamped) base cell, as the sort bins it.
    __device__ __forceinline__ unsigned baseBlock(const GridGeom &g, const Stencil &s, int &bx, int &by, int &bz)
    {
        bx = min(max(s.b[0], 0), max(g.n.x - 2, 0)) >> 2;
        by = min(max(s.b[1], 0), max(g.n.y - 2, 0)) >> 2;
        bz = min(max(s.b[2], 0), max(g.n.z - 2, 0)) >> 2;
        return g.blockBase + (unsigned)(bx + g.nb.x * (by + g.nb.y * bz));
    }

    __device__ __forceinline__ void loadM3(const float *planes, unsigned stride, unsigned i, M3 &m)
    {
#pragma unroll
        for (int k = 0; k < 9; ++k)
            m.m[k] = planes[k * stride + i];
    }
    __device__ __forceinline__ void storeM3(float *planes, unsigned stride, unsigned i, const M3 &m)
    {
#pragma unroll
        for (int k = 0; k < 9; ++k)
            planes[k * stride + i] = m.m[k];
    }

    // Per-thread asynchronous global -> shared copies (cp.async).  A thread stages its own
    // particle's streams, all in flight at once without holding registers, and waits for them with
    // stageWait; no other thread reads them, so no block barrier is needed.  Every thread that
    // issued copies waits before it exits.
    __device__ __forceinline__ void stage4(float *dst, const float *src)
    {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                     "l"(src)
                     : "memory");
    }
    __device__ __forceinline__ void stage16(float4 *dst, const float4 *src)
    {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                     "l"(src)
                     : "memory");
    }
    __device__ __forceinline__ void stageWait()
    {
        asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
    }

    __device__ __forceinline__ void loadShapes(ShapeRec *dst, const ShapeRec *src, int num)
    {
        const int words = num * (int)(sizeof(ShapeRec) / sizeof(float4));
        const float4 *s = reinterpret_cast<const float4 *>(src);
        float4 *d = reinterpret_cast<float4 *>(dst);
        for (int t = threadIdx.x; t < words; t += blockDim.x)
            d[t] = s[t];
    }

    // Records one binned particle of the calling lanes (active lanes `am`): its key, its rank among
    // the particles of its cell (arrival order), and the cell and block counts, with one atomic per
    // group of lanes sharing a cell or a block.
    __device__ __forceinline__ void binAggregated(unsigned am, unsigned lane, unsigned key, unsigned *__restrict__ blockCount,
                                                  unsigned *__restrict__ cellCount, unsigned *keyOut, unsigned *rankOut)
    {
        const unsigned lt = (1u << lane) - 1u;
        const unsigned cellPeers = __match_any_sync(am, key);
        const int cellLeader = __ffs(cellPeers) - 1;
        unsigned base = 0;
        if (key != kInvalidKey && (int)lane == cellLeader)
            base = atomicAdd(&cellCount[key], (unsigned)__popc(cellPeers));
        base = __shfl_sync(am, base, cellLeader);
        const unsigned blk = key == kInvalidKey ? kInvalidKey : key >> 6;
        const unsigned blkPeers = __match_any_sync(am, blk);
        if (blk != kInvalidKey && (int)lane == __ffs(blkPeers) - 1)
            atomicAdd(&blockCount[blk], (unsigned)__popc(blkPeers));
        if (keyOut)
        {
            *keyOut = key;
            *rankOut = base + (unsigned)__popc(cellPeers & lt);
        }
    }

    // Scene of a block (binary search over the scenes' block bases; scene 0 for one scene).
    __device__ __forceinline__ int sceneOfBlock(const SceneTable &sc, unsigned b)
    {
        int lo = 0, hi = sc.numScenes - 1;
        while (lo < hi)
        {
            const int mid = (lo + hi + 1) >> 1;
            if (sc.params[mid].g.blockBase <= b)
                lo = mid;
            else
                hi = mid - 1;
        }
        return lo;
    }

    // ---------------------------------------------------------------------------------------
    // 1. Shape table
    __global__ void k_gatherShapes(const __grid_constant__ StepParams p, SceneTable sc, const int *__restrict__ shapeIds, CrB200ShapeData sh,
                                   CrB200GeometryData ge, ShapeRec *__restrict__ out)
    {
        __shared__ int flags;
        __shared__ unsigned long long dynamic; // single scene: bit s = shape s is dynamic
        const int scene = blockIdx.x;
        const StepParams &sp = sc.numScenes > 1 ? sc.params[scene] : p;
        if (threadIdx.x == 0)
        {
            flags = 0;
            dynamic = 0ull;
        }
        __syncthreads();
        if (sc.numScenes == 1)
            for (int s = threadIdx.x; s < sp.numShapes && s < 64; s += blockDim.x)
                if (sh.type[shapeIds[sp.shapeBegin + s]] == S_DYNAMIC)
                    atomicOr(&dynamic, 1ull << s);
        __syncthreads();
        for (int s = threadIdx.x; s < sp.numShapes; s += blockDim.x)
        {
            const int t = sp.shapeBegin + s;
            ShapeRec r = makeShapeRec(shapeIds[t], sh, ge);
            if (sc.numScenes == 1 && s < 64 && r.kind == S_DYNAMIC)
                r.dynSlot = __popcll(dynamic & ((1ull << s) - 1ull)); // rank among the dynamic shapes
            out[t] = r;
            atomicOr(&flags, shapeFlagsOf(r));
        }
        __syncthreads();
        if (threadIdx.x == 0)
            sc.flags[scene] = (unsigned)flags;
    }

    // ---------------------------------------------------------------------------------------
    // 2. Bin: cell keys and warp-aggregated block histogram (rank = arrival order in its block).
    template <bool Multi>
    __global__ void k_bin(const __grid_constant__ StepParams p, SceneTable sc, bool ignoreMask, const float4 *__restrict__ xm,
                          const unsigned char *__restrict__ mask, unsigned *__restrict__ keys,
                          unsigned *__restrict__ ranks, unsigned *__restrict__ blockCount,
                          unsigned *__restrict__ cellCount, SortHeader *hdr)
    {
        if ((!Multi && hdr->recordsValid) || hdr->sortSkip)
            return; // the previous substep's G2P binned the particles (single scene, MLS), or the
                    // resident path keeps its order this call
        const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
        const unsigned lane = threadIdx.x & 31;
        const unsigned n = Multi ? sc.numParticles : p.numActive;
        unsigned key = kInvalidKey;
        bool ood = false;
        bool carried = false; // batch: binned by the previous G2P (scene without a slicer)
        if (i < n && (ignoreMask || mask[i]))
        {
            const unsigned short si = Multi ? sc.particleScene[i] : 0;
            carried = Multi && si != 0xFFFF && hdr->recordsValid && !(sc.flags[si] & SF_SLICER);
            if ((!Multi || si != 0xFFFF) && !carried)
            {
                const GridGeom &g = Multi ? sc.params[si].g : p.g;
                const float4 x = xm[i];
                const Stencil s = stencilOf(g, v3(x));
                if (s.finite)
                    key = cellKey(g, s, &ood);
                else
                    ood = true;
            }
        }
        const bool write = i < n && !carried;
        binAggregated(0xffffffffu, lane, key, blockCount, cellCount, write ? &keys[i] : nullptr, write ? &ranks[i] : nullptr);
        if (__any_sync(0xffffffffu, ood) && lane == 0)
            atomicOr(&hdr->status, CRB200_STATUS_OUT_OF_DOMAIN);
    }

    // ---------------------------------------------------------------------------------------
    // 3. Scan over blocks.  Tile t covers blocks [t*kScanTile, (t+1)*kScanTile).
    //    flags bit 0: block holds particles; bit 1: block holds nodes some particle touches
    //    (the block itself or one of its -x/-y/-z neighbours holds particles).
    __global__ void k_scanReduce(StepParams p, SceneTable sc, unsigned totalBlocks,
                                 const unsigned *__restrict__ blockCount, unsigned char *__restrict__ flags,
                                 uint3 *__restrict__ tileSums, const SortHeader *__restrict__ hdr)
    {
        if (hdr->sortSkip)
            return;
        unsigned sum = 0, act = 0, tch = 0;
        const unsigned b0 = blockIdx.x * kScanTile + threadIdx.x * (kScanTile / kScanThreads);
        for (int e = 0; e < kScanTile / kScanThreads; ++e)
        {
            const unsigned b = b0 + e;
            if (b >= totalBlocks)
                break;
            const GridGeom &g = sc.numScenes > 1 ? sc.params[sceneOfBlock(sc, b)].g : p.g;
            const unsigned lb = b - g.blockBase;
            const int bx = lb % g.nb.x, by = (lb / g.nb.x) % g.nb.y, bz = lb / (g.nb.x * g.nb.y);
            const unsigned c = blockCount[b];
            bool touched = false;
            for (int d = 0; d < 8 && !touched; ++d)
            {
                const int x = bx - (d & 1), y = by - ((d >> 1) & 1), z = bz - (d >> 2);
                if (x < 0 || y < 0 || z < 0)
                    continue;
                touched = blockCount[g.blockBase + x + g.nb.x * (y + g.nb.y * z)] > 0;
            }
            flags[b] = (unsigned char)((c > 0 ? 1 : 0) | (touched ? 2 : 0));
            sum += c;
            act += c > 0;
            tch += touched;
        }
        // block reduction
        __shared__ unsigned red[3][kScanThreads / 32];
        for (int o = 16; o > 0; o >>= 1)
        {
            sum += __shfl_down_sync(0xffffffffu, sum, o);
            act += __shfl_down_sync(0xffffffffu, act, o);
            tch += __shfl_down_sync(0xffffffffu, tch, o);
        }
        if ((threadIdx.x & 31) == 0)
        {
            red[0][threadIdx.x >> 5] = sum;
            red[1][threadIdx.x >> 5] = act;
            red[2][threadIdx.x >> 5] = tch;
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            uint3 t = make_uint3(0, 0, 0);
            for (int w = 0; w < kScanThreads / 32; ++w)
            {
                t.x += red[0][w];
                t.y += red[1][w];
                t.z += red[2][w];
            }
            tileSums[blockIdx.x] = t;
        }
    }

    // Exclusive scan of the tile sums (single CTA) + totals into the header.
    // A sorted total above the pair buffer's capacity (inconsistent block counts) empties the
    // block lists and raises CRB200_STATUS_BLOCK_OVERFLOW instead of letting later kernels run
    // past the buffers.
    __global__ void k_scanTiles(uint3 *__restrict__ tileSums, unsigned numTiles, SortHeader *hdr, unsigned capacity)
    {
        if (hdr->sortSkip)
            return;
        __shared__ uint3 carry;
        __shared__ uint3 warpTot[32];
        if (threadIdx.x == 0)
            carry = make_uint3(0, 0, 0);
        __syncthreads();
        for (unsigned base = 0; base < numTiles; base += blockDim.x)
        {
            const unsigned t = base + threadIdx.x;
            uint3 v = t < numTiles ? tileSums[t] : make_uint3(0, 0, 0);
            uint3 inc = v;
            const unsigned lane = threadIdx.x & 31, w = threadIdx.x >> 5;
            for (int o = 1; o < 32; o <<= 1)
            {
                const unsigned a = __shfl_up_sync(0xffffffffu, inc.x, o), b = __shfl_up_sync(0xffffffffu, inc.y, o),
                               c = __shfl_up_sync(0xffffffffu, inc.z, o);
                if (lane >= (unsigned)o)
                {
                    inc.x += a;
                    inc.y += b;
                    inc.z += c;
                }
            }
            if (lane == 31)
                warpTot[w] = inc;
            __syncthreads();
            if (w == 0)
            {
                uint3 x = lane < (blockDim.x >> 5) ? warpTot[lane] : make_uint3(0, 0, 0);
                for (int o = 1; o < 32; o <<= 1)
                {
                    const unsigned a = __shfl_up_sync(0xffffffffu, x.x, o), b = __shfl_up_sync(0xffffffffu, x.y, o),
                                   c = __shfl_up_sync(0xffffffffu, x.z, o);
                    if (lane >= (unsigned)o)
                    {
                        x.x += a;
                        x.y += b;
                        x.z += c;
                    }
                }
                warpTot[lane] = x; // inclusive over warps
            }
            __syncthreads();
            const uint3 wprev = w > 0 ? warpTot[w - 1] : make_uint3(0, 0, 0);
            const uint3 c = carry;
            if (t < numTiles)
                tileSums[t] = make_uint3(c.x + wprev.x + inc.x - v.x, c.y + wprev.y + inc.y - v.y, c.z + wprev.z + inc.z - v.z);
            __syncthreads();
            if (threadIdx.x == blockDim.x - 1)
            {
                const uint3 tot = warpTot[(blockDim.x >> 5) - 1];
                carry = make_uint3(c.x + tot.x, c.y + tot.y, c.z + tot.z);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0)
        {
            const bool over = carry.x > capacity;
            hdr->numSorted = over ? 0u : carry.x;
            hdr->numActiveBlocks = over ? 0u : carry.y;
            hdr->numTouchedBlocks = over ? 0u : carry.z;
            hdr->touchedNodes = 0;
            if (over)
                atomicOr(&hdr->status, CRB200_STATUS_BLOCK_OVERFLOW);
        }
    }

    __global__ void k_scanWrite(unsigned totalBlocks, const uint3 *__restrict__ tileOffsets,
                                unsigned *__restrict__ blockCount, const unsigned char *__restrict__ flags,
                                unsigned *__restrict__ blockStart, unsigned *__restrict__ activeList,
                                unsigned *__restrict__ touchedList, const SortHeader *__restrict__ hdr)
    {
        if (hdr->sortSkip)
            return;
        constexpr int per = kScanTile / kScanThreads;
        const unsigned b0 = blockIdx.x * kScanTile + threadIdx.x * per;
        unsigned cnt[per];
        unsigned char fl[per];
        unsigned sum = 0, act = 0, tch = 0;
#pragma unroll
        for (int e = 0; e < per; ++e)
        {
            const unsigned b = b0 + e;
            cnt[e] = b < totalBlocks ? blockCount[b] : 0;
            fl[e] = b < totalBlocks ? flags[b] : 0;
            sum += cnt[e];
            act += fl[e] & 1;
            tch += (fl[e] >> 1) & 1;
        }
        // block exclusive scan of (sum, act, tch)
        __shared__ uint3 warpTot[kScanThreads / 32];
        const unsigned lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        uint3 inc = make_uint3(sum, act, tch);
        for (int o = 1; o < 32; o <<= 1)
        {
            const unsigned a = __shfl_up_sync(0xffffffffu, inc.x, o), b = __shfl_up_sync(0xffffffffu, inc.y, o),
                           c = __shfl_up_sync(0xffffffffu, inc.z, o);
            if (lane >= (unsigned)o)
            {
                inc.x += a;
                inc.y += b;
                inc.z += c;
            }
        }
        if (lane == 31)
            warpTot[w] = inc;
        __syncthreads();
        uint3 wp = make_uint3(0, 0, 0);
        for (unsigned k = 0; k < w; ++k)
        {
            wp.x += warpTot[k].x;
            wp.y += warpTot[k].y;
            wp.z += warpTot[k].z;
        }
        const uint3 to = tileOffsets[blockIdx.x];
        unsigned s = to.x + wp.x + inc.x - sum, a = to.y + wp.y + inc.y - act, t = to.z + wp.z + inc.z - tch;
#pragma unroll
        for (int e = 0; e < per; ++e)
        {
            const unsigned b = b0 + e;
            if (b >= totalBlocks)
                break;
            blockStart[b] = s;
            s += cnt[e];
            if (fl[e] & 1)
                activeList[a++] = b;
            if (fl[e] & 2)
                touchedList[t++] = b;
            blockCount[b] = 0;
            if (b == totalBlocks - 1)
                blockStart[totalBlocks] = s;
        }
    }

    // ---------------------------------------------------------------------------------------
    // 4. Scatter (local cell, id) into the block segments.
    __global__ void k_scatter(unsigned numActive, const unsigned *__restrict__ keys, const unsigned *__restrict__ ranks,
                              const unsigned *__restrict__ cellStart, unsigned *__restrict__ sortedIds,
                              unsigned capacity, const SortHeader *__restrict__ hdr)
    {
        const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= numActive || hdr->sortSkip)
            return;
        const unsigned key = keys[i];
        if (key == kInvalidKey)
            return;
        const unsigned slot = cellStart[key] + ranks[i];
        if (slot < capacity) // always, unless the block counts were inconsistent (flagged by k_scanTiles)
            sortedIds[slot] = i;
    }

    // Absolute start of every cell of the active blocks (one warp per block, lane l scanning cells l
    // and l + 32): the block's start plus the exclusive prefix of its cell counts, which are cleared
    // for the next binning.
    // Deterministic substeps: each cell's slots hold its particle ids in ascending order (the
    // scatter places them in arrival order).  One 64-thread CTA per active block: the block's ids
    // go to shared memory (coalesced), thread c insertion-sorts cell c's segment, and they go back;
    // a block larger than the buffer sorts in place in global memory.
    constexpr unsigned kCellOrderCap = 2048;
    __global__ void __launch_bounds__(64) k_cellOrder(const SortHeader *__restrict__ hdr,
                                                      const unsigned *__restrict__ activeList,
                                                      const unsigned *__restrict__ blockStart,
                                                      const unsigned *__restrict__ cellStart,
                                                      unsigned *__restrict__ sortedIds)
    {
        __shared__ unsigned sIds[kCellOrderCap];
        const unsigned tid = threadIdx.x, nAct = hdr->numActiveBlocks;
        for (unsigned ab = blockIdx.x; ab < nAct; ab += gridDim.x)
        {
            const unsigned b = activeList[ab], start = blockStart[b], cnt = blockStart[b + 1] - start;
            const unsigned s = cellStart[b * 64u + tid] - start;
            const unsigned e = (tid < 63u ? cellStart[b * 64u + tid + 1u] : blockStart[b + 1]) - start;
            unsigned *ids = cnt <= kCellOrderCap ? sIds : sortedIds + start;
            if (cnt <= kCellOrderCap)
            {
                for (unsigned t = tid; t < cnt; t += 64u)
                    sIds[t] = sortedIds[start + t];
                __syncthreads();
            }
            for (unsigned i = s + 1; i < e; ++i)
            {
                const unsigned v = ids[i];
                unsigned j = i;
                while (j > s && ids[j - 1] > v)
                {
                    ids[j] = ids[j - 1];
                    --j;
                }
                ids[j] = v;
            }
            if (cnt <= kCellOrderCap)
            {
                __syncthreads();
                for (unsigned t = tid; t < cnt; t += 64u)
                    sortedIds[start + t] = sIds[t];
                __syncthreads();
            }
        }
    }

    __global__ void __launch_bounds__(256) k_cellStarts(const SortHeader *__restrict__ hdr,
                                                        const unsigned *__restrict__ activeList,
                                                        const unsigned *__restrict__ blockStart,
                                                        unsigned *__restrict__ cellCount, unsigned *__restrict__ cellStart)
    {
        if (hdr->sortSkip)
            return;
        const unsigned lane = threadIdx.x & 31;
        const unsigned nWarps = (gridDim.x * blockDim.x) >> 5;
        const unsigned nAct = hdr->numActiveBlocks;
        for (unsigned ab = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ab < nAct; ab += nWarps)
        {
            const unsigned b = activeList[ab];
            const unsigned c0 = b * 64u + lane, c1 = c0 + 32u;
            const unsigned v0 = cellCount[c0], v1 = cellCount[c1];
            cellCount[c0] = 0u;
            cellCount[c1] = 0u;
            unsigned i0 = v0, i1 = v1;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1)
            {
                const unsigned y0 = __shfl_up_sync(0xffffffffu, i0, o), y1 = __shfl_up_sync(0xffffffffu, i1, o);
                if (lane >= (unsigned)o)
                {
                    i0 += y0;
                    i1 += y1;
                }
            }
            const unsigned firstHalf = __shfl_sync(0xffffffffu, i0, 31);
            const unsigned bs = blockStart[b];
            cellStart[c0] = bs + i0 - v0;
            cellStart[c1] = bs + firstHalf + i1 - v1;
        }
    }

}
#include "p2g_cells.cuh"
namespace crb200
{
    // Deterministic P2G: a node's sum over the 6x6x6 tiles of the active cell blocks that cover it
    // (its own block and, for the first two nodes along an axis, the block below), in a fixed order
    // of (dz, dy, dx), then `rest` (what per-particle atomics added to the node).
    __device__ __forceinline__ float4 gatherTiles(const GridGeom &g, const float4 *__restrict__ tiles,
                                                  const unsigned char *__restrict__ flags, int bx, int by, int bz,
                                                  unsigned l, float4 rest)
    {
        const int lx = l & 3, ly = (l >> 2) & 3, lz = l >> 4;
        // all loads first (source d = 4 dz + 2 dy + dx), then the sum in that order
        float4 v[8];
#pragma unroll
        for (int d = 0; d < 8; ++d)
        {
            const int dx = d & 1, dy = (d >> 1) & 1, dz = d >> 2;
            v[d] = make_float4(0.f, 0.f, 0.f, 0.f);
            if ((dx && (lx >= 2 || bx == 0)) || (dy && (ly >= 2 || by == 0)) || (dz && (lz >= 2 || bz == 0)))
                continue;
            const unsigned c = g.blockBase + (unsigned)(bx - dx) + g.nb.x * ((unsigned)(by - dy) + g.nb.y * (unsigned)(bz - dz));
            if (!(__ldg(&flags[c]) & 1u))
                continue;
            const int t = (lx + 4 * dx) + kTileEdge * ((ly + 4 * dy) + kTileEdge * (lz + 4 * dz));
            v[d] = tiles[(size_t)c * kTileNodes + t];
        }
        float4 s = v[0];
#pragma unroll
        for (int d = 1; d < 8; ++d)
        {
            s.x += v[d].x;
            s.y += v[d].y;
            s.z += v[d].z;
            s.w += v[d].w;
        }
        s.x += rest.x;
        s.y += rest.y;
        s.z += rest.z;
        s.w += rest.w;
        return s;
    }

    // 7. Grid update over touched blocks (mls_mpm_algorithm.h:243-294 and its PB / standard twins).
    //    Multi: the touched blocks belong to many scenes; each block reads its scene's parameters
    //    and shapes from global memory (single scene: kernel arguments and shared memory).
    //    Det >= 1: coupling momentum of the first kDetSlots dynamic shapes is summed per 4x4x4 block
    //    in a fixed order and written to detPartials[(block * kDetSlots + slot) * 2 + {0: force,
    //    1: torque}] (bit `block` of detMask set) for k_coupleReduce, instead of float atomics into
    //    the shapes' force and torque.
    //    Det == 2: the P2G grid comes from the cell blocks' tiles (k_accumulate<.., true>): each
    //    node sums the tiles that cover it in a fixed order (gatherTiles), then what per-particle
    //    atomics left in gridA (particles whose stencil leaves the grid).
    template <bool Multi, int Det>
    __global__ void __launch_bounds__(256) k_gridUpdate(const __grid_constant__ StepParams p0, SceneTable sc, const SortHeader *__restrict__ hdr,
                                                        const unsigned *__restrict__ touchedList,
                                                        const ShapeRec *__restrict__ shapeTable, SdfPtrs sdf,
                                                        float4 *__restrict__ gridA, float4 *__restrict__ gridF,
                                                        float4 *__restrict__ gridV, float4 *coupleForce,
                                                        float4 *coupleTorque, bool clearA,
                                                        unsigned long long *__restrict__ blockShapeMask,
                                                        float4 *__restrict__ saveA, float4 *__restrict__ saveV,
                                                        float4 *__restrict__ detPartials, unsigned *__restrict__ detMask,
                                                        unsigned detMaskWords,
                                                        const float4 *__restrict__ tiles, const float4 *__restrict__ tilesF,
                                                        const unsigned char *__restrict__ blockFlags,
                                                        unsigned *__restrict__ touchedFlag = nullptr)
    {
        // touchedFlag (resident path): the block's "already listed" flag, cleared as it is consumed
        __shared__ ShapeRec sh[Multi ? 1 : kMaxShapes];
        __shared__ unsigned sTouched;
        // Det (single scene): one row of coupling sums per thread.  A batch keeps the coupling
        // atomics: its tiles make the particle state reproducible, not the shapes' force sums.
        constexpr bool kRows = Det > 0 && !Multi;
        __shared__ float sCouple[kRows ? 256 : 1][kDetSlots * 6];
        if (threadIdx.x == 0)
            sTouched = 0;
        if (!Multi && p0.numShapes > 0)
            loadShapes(sh, shapeTable, p0.numShapes);
        __syncthreads();
        const unsigned nT = hdr->numTouchedBlocks;
        const bool withForce = p0.solverType == CRB200_SOLVER_GPU_STANDARD;
        const unsigned perCta = blockDim.x / 64;
        using Couple = typename std::conditional<kRows, CoupleRow, CoupleAtomic>::type;
        if constexpr (kRows)
            for (int c = 0; c < kDetSlots * 6; ++c)
                sCouple[threadIdx.x][c] = 0.f;
        for (unsigned base = blockIdx.x * perCta; base < nT; base += gridDim.x * perCta)
        {
            const unsigned bi = base + threadIdx.x / 64;
            Couple couple;
            if constexpr (kRows)
                couple = CoupleRow{sCouple[threadIdx.x], CoupleAtomic{coupleForce, coupleTorque}, false};
            else
                couple = CoupleAtomic{coupleForce, coupleTorque};
            unsigned b = 0;
            // one node of block touchedList[bi]; leaves early where the reference's update returns
            do
            {
                if (bi >= nT)
                    break;
                b = touchedList[bi];
                if (touchedFlag != nullptr && (threadIdx.x & 63) == 0)
                    touchedFlag[b] = 0u;
                const StepParams &p = Multi ? sc.params[sceneOfBlock(sc, b)] : p0;
                const GridGeom &g = p.g;
                const ShapeRec *shp = Multi ? shapeTable + p.shapeBegin : sh;
                const unsigned l = threadIdx.x & 63;
                const unsigned lb = b - g.blockBase;
                const int bx = lb % g.nb.x, by = (lb / g.nb.x) % g.nb.y, bz = lb / (g.nb.x * g.nb.y);
                // shapes that can reach this block's region: one test per shape and warp instead of
                // one per node, and the particle mask for G2P / PB-MPM integration
                const BlockRegion region = blockRegion(g, bx, by, bz);
                unsigned long long nodeMask = ~0ull;
                if (p.numShapes > 0)
                {
                    V3 bc;
                    float bR;
                    regionBall(region, bc, bR);
                    unsigned long long partMask;
                    regionShapeMasks(shp, p.numShapes, bc, bR, nodeMask, partMask);
                    if (l == 0)
                        blockShapeMask[b] = partMask;
                }
                const int i = 4 * bx + (l & 3), j = 4 * by + ((l >> 2) & 3), k = 4 * bz + (l >> 4);
                if (!inGrid(g, i, j, k))
                    break;
                const unsigned a = b * 64u + l;
                float4 acc = gridA[a];
                if (clearA)
                    gridA[a] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (Det == 2)
                    acc = gatherTiles(g, tiles, blockFlags, bx, by, bz, l, acc);
                if (saveA)
                    saveA[a] = acc; // the adjoint's tape of this substep's P2G grid
                float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
                if (withForce)
                {
                    f = gridF[a];
                    gridF[a] = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (Det == 2)
                        f = gatherTiles(g, tilesF, blockFlags, bx, by, bz, l, f);
                }
                {
                    // nodes that received mass (roofline bookkeeping): a shared counter per CTA
                    const unsigned am = __activemask();
                    const unsigned hit = __ballot_sync(am, acc.w > 0.f);
                    if ((threadIdx.x & 31) == (unsigned)(__ffs(am) - 1) && hit)
                        atomicAdd(&sTouched, (unsigned)__popc(hit));
                }
                if (acc.w < p.cutoff)
                {
                    gridV[a] = acc; // light nodes keep momentum, which G2P then reads (reference Q2)
                    if (saveV)
                        saveV[a] = acc;
                    break;
                }
                if (withForce)
                {
                    acc.x += f.x * p.dt;
                    acc.y += f.y * p.dt;
                    acc.z += f.z * p.dt;
                }
                V3 v = v3(acc.x / acc.w, acc.y / acc.w, acc.z / acc.w);
                V3 pos = v3((float)i * g.dx, (float)j * g.dx, (float)k * g.dx) + v3(g.gmin.x, g.gmin.y, g.gmin.z);
                pos = pos + v * p.dt;
                if (p.numShapes > 0)
                    rigidContact<false>(v, acc.w, pos, shp, p.numShapes, sdf, p.contactModel == 1, couple,
                                        region.contains(pos) ? nodeMask : ~0ull);
                if (i < 2 || i > g.n.x - 3)
                    v.x = 0.f;
                if (j < 2 || j > g.n.y - 3)
                    v.y = 0.f;
                if (k < 2 || k > g.n.z - 3)
                    v.z = 0.f;
                gridV[a] = make_float4(v.x, v.y, v.z, acc.w);
                if (saveV)
                    saveV[a] = make_float4(v.x, v.y, v.z, acc.w);
            } while (false);
            if constexpr (kRows)
            {
                // block sums in a fixed order: thread c < 24 of each 64-thread group adds column c
                // of the group's rows in row order, writes it and clears the column
                if (__syncthreads_or(couple.any))
                {
                    const unsigned l = threadIdx.x & 63, g0 = threadIdx.x - l;
                    if (l < kDetSlots * 6 && bi < nT)
                    {
                        float t = 0.f;
                        for (int r = 0; r < 64; ++r)
                        {
                            t += sCouple[g0 + r][l];
                            sCouple[g0 + r][l] = 0.f;
                        }
                        const int slot = l / 6, c = l % 6;
                        float *dst = reinterpret_cast<float *>(&detPartials[((size_t)b * kDetSlots + slot) * 2 + c / 3]);
                        dst[c % 3] = t;
                        if (l == 0)
                        {
                            atomicOr(&detMask[b >> 5], 1u << (b & 31)); // the block holds partials
                            atomicOr(&detMask[detMaskWords], 1u);        // and so does the substep
                        }
                    }
                    __syncthreads();
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && sTouched)
            atomicAdd(&const_cast<SortHeader *>(hdr)->touchedNodes, sTouched);
    }

    // Deterministic coupling reduction (one CTA): the blocks flagged in detMask, each thread taking
    // mask words t, t + 256, ... and their blocks in ascending order, then a fixed tree over the
    // threads; the sums are added to the dynamic shapes' force and torque.  Mask words and partials
    // are zeroed once read.
    __global__ void __launch_bounds__(256) k_coupleReduce(unsigned numMaskWords, unsigned *__restrict__ detMask,
                                                          float4 *__restrict__ detPartials,
                                                          const ShapeRec *__restrict__ shapeTable, int numShapes,
                                                          float4 *force, float4 *torque)
    {
        __shared__ float sSum[256][kDetSlots * 6 + 1];
        // word numMaskWords is set when any block holds partials (not on substeps without coupling)
        if (detMask[numMaskWords] == 0u)
            return;
        __syncthreads();
        if (threadIdx.x == 0)
            detMask[numMaskWords] = 0u;
        float t[kDetSlots * 6];
#pragma unroll
        for (int c = 0; c < kDetSlots * 6; ++c)
            t[c] = 0.f;
        for (unsigned w = threadIdx.x; w < numMaskWords; w += blockDim.x)
        {
            unsigned m = detMask[w];
            if (!m)
                continue;
            detMask[w] = 0u;
            while (m)
            {
                const unsigned b = w * 32u + (unsigned)(__ffs(m) - 1);
                m &= m - 1u;
#pragma unroll
                for (int s = 0; s < kDetSlots; ++s)
                {
                    const size_t e = ((size_t)b * kDetSlots + s) * 2;
                    const float4 f = detPartials[e], q = detPartials[e + 1];
                    t[6 * s + 0] += f.x, t[6 * s + 1] += f.y, t[6 * s + 2] += f.z;
                    t[6 * s + 3] += q.x, t[6 * s + 4] += q.y, t[6 * s + 5] += q.z;
                    detPartials[e] = make_float4(0.f, 0.f, 0.f, 0.f);
                    detPartials[e + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
        }
#pragma unroll
        for (int c = 0; c < kDetSlots * 6; ++c)
            sSum[threadIdx.x][c] = t[c];
        __syncthreads();
        for (int h = blockDim.x / 2; h > 0; h >>= 1)
        {
            if (threadIdx.x < (unsigned)h)
                for (int c = 0; c < kDetSlots * 6; ++c)
                    sSum[threadIdx.x][c] += sSum[threadIdx.x + h][c];
            __syncthreads();
        }
        if (threadIdx.x == 0 && force && torque)
            for (int s = 0; s < numShapes; ++s)
            {
                const int slot = shapeTable[s].dynSlot;
                if (slot < 0 || slot >= kDetSlots)
                    continue;
                const int id = shapeTable[s].id;
                const float *v = sSum[0] + 6 * slot;
                force[id].x += v[0], force[id].y += v[1], force[id].z += v[2];
                torque[id].x += v[3], torque[id].y += v[4], torque[id].z += v[5];
            }
    }

    // 8. G2P in particle order.  Mode 0 MLS (mls_mpm_algorithm.h:296-390), 1 PB
    //    (pb_mpm_algorithm.h:286-361, v and C only), 2 standard (standard_mpm_algorithm.h:274-352).
    //    Node addresses are separable in the block-major layout (addr = AX[i] + AY[j] + AZ[k]); a
    //    particle whose stencil lies inside the grid skips all per-node bounds tests.  The APIC
    //    matrix 4/dx sum_n d_r (w v)_c is accumulated as 4/dx dx (sum_n ijk_r (w v)_c - fx_r sum_n (w v)_c).
    // One node of the G2P gather: v += w v_n and the APIC moments (Modes 0/1) or grad v (Mode 2).
    template <int Mode>
    __device__ __forceinline__ void g2pNode(int a, int b, int c, V3 nv, const float w[3][3], const float dw[3][3], V3 &S,
                                            float T[9])
    {
        const float wt = w[a][0] * w[b][1] * w[c][2];
        if (Mode == 2)
        {
            S = S + nv * wt;
            const float gw[3] = {dw[a][0] * w[b][1] * w[c][2], w[a][0] * dw[b][1] * w[c][2], w[a][0] * w[b][1] * dw[c][2]};
            // gradientVelocity += gw.outerProduct(nv): M(r, c) = gw_c * nv_r
#pragma unroll
            for (int cc = 0; cc < 3; ++cc)
            {
                T[cc * 3 + 0] += gw[cc] * nv.x;
                T[cc * 3 + 1] += gw[cc] * nv.y;
                T[cc * 3 + 2] += gw[cc] * nv.z;
            }
        }
        else
        {
            const V3 wv = nv * wt;
            S = S + wv;
            if (a)
            {
                T[0] += (float)a * wv.x;
                T[1] += (float)a * wv.y;
                T[2] += (float)a * wv.z;
            }
            if (b)
            {
                T[3] += (float)b * wv.x;
                T[4] += (float)b * wv.y;
                T[5] += (float)b * wv.z;
            }
            if (c)
            {
                T[6] += (float)c * wv.x;
                T[7] += (float)c * wv.y;
                T[8] += (float)c * wv.z;
            }
        }
    }

    // G2P gather for a stencil that crosses the grid boundary or has cut nodes (out of line: rare).
    // Everything is passed and returned by value so that the caller's weights stay in registers.
    struct G2PWeights
    {
        float w[3][3], dw[3][3];
    };
    struct G2PMoments
    {
        V3 S;
        float T[9];
    };

    template <int Mode>
    __device__ __noinline__ G2PMoments g2pGatherGeneral(GridGeom g, Stencil st, V3 x, V3 vk, unsigned msk, G2PWeights W,
                                                        const ShapeRec *sh, int numShapes, SdfPtrs sdf,
                                                        const float4 *__restrict__ gridV)
    {
        G2PMoments r;
        r.S = v3(0.f, 0.f, 0.f);
#pragma unroll
        for (int e = 0; e < 9; ++e)
            r.T[e] = 0.f;
#pragma unroll 1
        for (int n = 0; n < 27; ++n)
        {
            const int a = n / 9, b = (n / 3) % 3, c = n % 3;
            const int ni = st.b[0] + a, nj = st.b[1] + b, nk = st.b[2] + c;
            if (!inGrid(g, ni, nj, nk))
                continue;
            V3 nv = v3(__ldg(&gridV[nodeAddr(g, ni, nj, nk)]));
            if (Mode != 2 && ((msk >> n) & 1u))
            {
                const V3 d = v3(ex::mul(ex::sub((float)a, st.fx.x), g.dx), ex::mul(ex::sub((float)b, st.fx.y), g.dx),
                                ex::mul(ex::sub((float)c, st.fx.z), g.dx));
                V3 nrm;
                if (differentSides(x, ex::add(x, d), sh, numShapes, sdf, &nrm))
                    nv = vk - nrm * dot(vk, nrm) * 2.0f;
            }
            g2pNode<Mode>(a, b, c, nv, W.w, W.dw, r.S, r.T);
        }
        return r;
    }

    //    records != nullptr (MLS, one scene): also build the next substep's P2G record of the updated
    //    particle (what k_record would compute from the stored state) unless a slicer is present,
    //    and mark the records valid; particles whose new stencil leaves the grid are scattered into
    //    the (cleared) accumulation grid here, as k_record does.
    template <int Mode, bool Multi>
    __global__ void __launch_bounds__(128, Mode == 1 ? 4 : ((Mode == 0 && !Multi) ? 7 : 6)) k_g2p(const __grid_constant__ StepParams p0, SceneTable sc, float4 *xm,
                                                 float4 *vel, const unsigned char *__restrict__ mask,
                                                 float *F, float *Cm, unsigned stride,
                                                 const ShapeRec *__restrict__ shapeTable, SdfPtrs sdf,
                                                 const float4 *__restrict__ gridV, const unsigned *__restrict__ cutMasks,
                                                 unsigned *status, const float4 *__restrict__ matParams,
                                                 const int *__restrict__ matType, const float *__restrict__ V0,
                                                 float4 *__restrict__ records, float4 *__restrict__ gridA,
                                                 SortHeader *hdr, unsigned *__restrict__ keys,
                                                 unsigned *__restrict__ ranks, unsigned *__restrict__ blockCount,
                                                 unsigned *__restrict__ cellCount,
                                                 const unsigned long long *__restrict__ blockShapeMask,
                                                 float4 *xo, float4 *vo, float *Fo, float *Co, bool lean)
    {
        // Modes 0 and 2 write the updated state to xo, vo, Fo, Co: the input arrays themselves in an
        // ordinary substep, the next tape slot in the adjoint's replay (which keeps its input).
        // Inputs and outputs may therefore alias, so none of xm, vel, F, Cm, xo, vo, Fo, Co is
        // declared __restrict__; each thread reads its own particle before it writes it.
        // lean (MLS, a substep of a call but its last): a particle whose next P2G record is written
        // here does not write its velocity and C, which only that record carries forward; the
        // call's last substep writes them for the caller and the next call.
        // One scene: all or nothing (no slicer in the scene).  Batch: per particle, for the scenes
        // without a slicer (k_bin / k_record skip exactly those particles in the next substep).
        if (Mode == 1 && blockIdx.x == 0 && threadIdx.x == 0)
            hdr->pbRecordsValid = records != nullptr ? 1u : 0u; // read only by later launches
        constexpr bool kRecords = Mode == 0;
        const bool writeRecords =
            kRecords && records != nullptr && (Multi || !(p0.numShapes > 0 && (sc.flags[0] & SF_SLICER)));
        if (writeRecords && blockIdx.x == 0 && threadIdx.x == 0)
            hdr->recordsValid = 1u; // read only by later launches
        __shared__ ShapeRec sh[Multi ? 1 : kMaxShapes];
        if (!Multi && p0.numShapes > 0)
        {
            loadShapes(sh, shapeTable, p0.numShapes);
            __syncthreads();
        }
        const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= (Multi ? sc.numParticles : p0.numActive) || !mask[i])
            return;
        const unsigned si = Multi ? sc.particleScene[i] : 0u;
        if (Multi && si == 0xFFFFu)
            return;
        const StepParams &p = Multi ? sc.params[si] : p0;
        const GridGeom &g = p.g;
        const ShapeRec *shp = Multi ? shapeTable + p.shapeBegin : sh;
        const bool slicers = Mode != 2 && p.numShapes > 0 && (sc.flags[si] & SF_SLICER);
        // F (and for the next record the material and V0) are used only after the node gathers:
        // start their DRAM reads into L2 now, so that they arrive while the gathers wait, without
        // holding registers across them
        if (Mode != 1)
        {
#pragma unroll
            for (int e = 0; e < 9; ++e)
                asm volatile("prefetch.global.L2 [%0];" ::"l"(F + (size_t)e * stride + i));
            if (Mode == 0 && records != nullptr)
            {
                asm volatile("prefetch.global.L2 [%0];" ::"l"(matParams + i));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(V0 + i));
            }
        }
        const float4 x4 = xm[i];
        const V3 x = v3(x4);
        const Stencil st = stencilOf(g, x);
        float w[3][3], dw[3][3];
        weights(st.fx, w);
        if (Mode == 2)
            weightGrads(st.fx, dw);
        const unsigned msk = slicers ? cutMasks[i] : 0u;
        V3 vk = v3(0.f, 0.f, 0.f);
        if (msk)
        {
            vk = v3(vel[i]);
            if (Mode == 0)
                vk = vk + v3(p.gravity) * p.dt; // the velocity P2G kicked (mls_mpm_algorithm.h:178)
        }
        V3 S = v3(0.f, 0.f, 0.f);
        float T[9]; // Modes 0/1: T[3r + c] = sum ijk_r (w v)_c; Mode 2: grad v, column-major
#pragma unroll
        for (int e = 0; e < 9; ++e)
            T[e] = 0.f;
        if (st.finite)
        {
            const bool interior = st.b[0] >= 0 && st.b[0] <= g.n.x - 3 && st.b[1] >= 0 && st.b[1] <= g.n.y - 3 &&
                                  st.b[2] >= 0 && st.b[2] <= g.n.z - 3;
            if (interior && msk == 0u)
            {
                unsigned AX[3], AY[3], AZ[3];
#pragma unroll
                for (int e = 0; e < 3; ++e)
                {
                    const int xi = st.b[0] + e, yi = st.b[1] + e, zi = st.b[2] + e;
                    AX[e] = g.blockBase * 64u + (unsigned)(((xi >> 2) << 6) + (xi & 3));
                    AY[e] = (unsigned)(((g.nb.x * (yi >> 2)) << 6) + 4 * (yi & 3));
                    AZ[e] = (unsigned)(((g.nb.x * g.nb.y * (zi >> 2)) << 6) + 16 * (zi & 3));
                }
                if (Mode == 2)
                {
#pragma unroll
                    for (int a = 0; a < 3; ++a)
#pragma unroll
                        for (int b = 0; b < 3; ++b)
#pragma unroll
                            for (int c = 0; c < 3; ++c)
                                g2pNode<Mode>(a, b, c, v3(__ldg(&gridV[AX[a] + AY[b] + AZ[c]])), w, dw, S, T);
                }
                else
                {
                    // The weight is a product of 1D factors, so v and the offset moments contract
                    // axis by axis: over c (Z = sum w_c V, Zc = sum c w_c V), then b, then a.
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                    {
                        V3 Y = v3(0.f, 0.f, 0.f), Yb = v3(0.f, 0.f, 0.f), Yc = v3(0.f, 0.f, 0.f);
#pragma unroll
                        for (int b = 0; b < 3; ++b)
                        {
                            const unsigned ab = AX[a] + AY[b];
                            const V3 v0 = v3(__ldg(&gridV[ab + AZ[0]])), v1 = v3(__ldg(&gridV[ab + AZ[1]])),
                                     v2 = v3(__ldg(&gridV[ab + AZ[2]]));
                            const V3 Zc = fma3(v2, 2.f * w[2][2], mul3(v1, w[1][2]));
                            const V3 Z = fma3(v2, w[2][2], fma3(v1, w[1][2], mul3(v0, w[0][2])));
                            Y = fma3(Z, w[b][1], Y);
                            if (b)
                                Yb = fma3(Z, (float)b * w[b][1], Yb);
                            Yc = fma3(Zc, w[b][1], Yc);
                        }
                        const V3 wY = Y * w[a][0];
                        S = S + wY;
                        if (a)
                        {
                            T[0] += (float)a * wY.x;
                            T[1] += (float)a * wY.y;
                            T[2] += (float)a * wY.z;
                        }
                        T[3] += w[a][0] * Yb.x;
                        T[4] += w[a][0] * Yb.y;
                        T[5] += w[a][0] * Yb.z;
                        T[6] += w[a][0] * Yc.x;
                        T[7] += w[a][0] * Yc.y;
                        T[8] += w[a][0] * Yc.z;
                    }
                }
            }
            else
            {
                G2PWeights W;
#pragma unroll
                for (int q = 0; q < 3; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                    {
                        W.w[q][d] = w[q][d];
                        W.dw[q][d] = Mode == 2 ? dw[q][d] : 0.f;
                    }
                const G2PMoments r = g2pGatherGeneral<Mode>(g, st, x, vk, msk, W, shp, p.numShapes, sdf, gridV);
                S = r.S;
#pragma unroll
                for (int e = 0; e < 9; ++e)
                    T[e] = r.T[e];
            }
        }
        M3 Cn;
        if (Mode == 2)
        {
#pragma unroll
            for (int e = 0; e < 9; ++e)
                Cn.m[e] = T[e];
        }
        else
        {
            const float s4 = 4.f * g.invDx * g.dx;
            const float fx[3] = {st.fx.x, st.fx.y, st.fx.z};
            const float Sv[3] = {S.x, S.y, S.z};
            // C(r, c) = 4/dx sum d_r (w v)_c, column-major m[3c + r]
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    Cn.m[3 * c + r] = s4 * (T[3 * r + c] - fx[r] * Sv[c]);
        }
        const V3 va = S;
        if (Mode == 1)
        {
            vel[i] = make_float4(va.x, va.y, va.z, 0.f);
            storeM3(Cm, stride, i, Cn);
            if (records)
            {
                // the next iteration's P2G record: the material constraint on the new C (which
                // stores the relaxed C) and the record, as k_record would build them
                RawParticle raw;
                raw.x4 = x4;
                raw.v4 = make_float4(va.x, va.y, va.z, 0.f);
                raw.mp = matParams[i];
                raw.mt = matType[i];
                M3 Fp;
                loadM3(F, stride, i, Fp);
#pragma unroll
                for (int e = 0; e < 9; ++e)
                {
                    raw.F[e] = Fp.m[e];
                    raw.C[e] = Cn.m[e];
                }
                raw.v0 = 0.f;
                float rec[kRec];
                if (!buildRecord<1>(p, i, raw, Cm, stride, msk, true, gridA, nullptr, &hdr->fp64Fallbacks, rec))
                {
#pragma unroll
                    for (int e = 0; e < kRec; ++e)
                        rec[e] = 0.f;
                }
                float4 *out = records + 4ull * i;
                out[0] = make_float4(rec[0], rec[1], rec[2], rec[3]);
                out[1] = make_float4(rec[4], rec[5], rec[6], rec[7]);
                out[2] = make_float4(rec[8], rec[9], rec[10], rec[11]);
                out[3] = make_float4(rec[12], rec[13], rec[14], rec[15]);
            }
            return;
        }
        V3 xn = x + va * p.dt;
        xn = v3(fminf(fmaxf(xn.x, g.gmin.x), g.gmax.x), fminf(fmaxf(xn.y, g.gmin.y), g.gmax.y),
                fminf(fmaxf(xn.z, g.gmin.z), g.gmax.z));
        V3 vn = va;
        if (p.numShapes > 0)
        {
            int bx, by, bz;
            const unsigned blk = baseBlock(g, st, bx, by, bz);
            const bool near = blockRegion(g, bx, by, bz).contains(xn);
            CoupleAtomic noCouple{nullptr, nullptr}; // particle push-out exchanges no momentum
            rigidContact<true>(vn, x4.w, xn, shp, p.numShapes, sdf, false, noCouple,
                               near ? blockShapeMask[blk] : ~0ull);
        }
        M3 Fp, Mu;
        loadM3(F, stride, i, Fp);
#pragma unroll
        for (int e = 0; e < 9; ++e)
            Mu.m[e] = ((e % 4) == 0 ? 1.f : 0.f) + Cn.m[e] * p.dt;
        Fp = matmul(Mu, Fp);
        const bool carried = kRecords && writeRecords && !(Multi && (sc.flags[si] & SF_SLICER));
        xo[i] = make_float4(xn.x, xn.y, xn.z, x4.w);
        if (!(lean && carried))
            vo[i] = make_float4(vn.x, vn.y, vn.z, 0.f);
        storeM3(Fo, stride, i, Fp);
        if (Mode == 0 && !(lean && carried))
            storeM3(Co, stride, i, Cn);
        if (!(isfinite(xn.x) && isfinite(xn.y) && isfinite(xn.z) && isfinite(vn.x) && isfinite(vn.y) && isfinite(vn.z)))
            atomicOr(status, CRB200_STATUS_NAN_STATE);
        if (carried)
        {
            RawParticle raw;
            raw.x4 = make_float4(xn.x, xn.y, xn.z, x4.w);
            raw.v4 = make_float4(vn.x, vn.y, vn.z, 0.f);
            raw.mp = matParams[i];
            raw.mt = matType[i];
#pragma unroll
            for (int e = 0; e < 9; ++e)
            {
                raw.F[e] = Fp.m[e];
                raw.C[e] = Cn.m[e];
            }
            raw.v0 = V0[i];
            float rec[kRec];
            if (!buildRecord<0>(p, i, raw, nullptr, stride, 0u, true, gridA, nullptr, nullptr, rec))
            {
#pragma unroll
                for (int e = 0; e < kRec; ++e)
                    rec[e] = 0.f;
            }
            float4 *out = records + 4ull * i;
            out[0] = make_float4(rec[0], rec[1], rec[2], rec[3]);
            out[1] = make_float4(rec[4], rec[5], rec[6], rec[7]);
            out[2] = make_float4(rec[8], rec[9], rec[10], rec[11]);
            out[3] = make_float4(rec[12], rec[13], rec[14], rec[15]);
            // binning of the new position for the next substep (what k_bin computes); the lanes
            // still running aggregate their block histogram updates
            const Stencil sn = stencilOf(g, xn);
            bool ood = false;
            unsigned key = kInvalidKey;
            if (sn.finite)
                key = cellKey(g, sn, &ood);
            else
                ood = true;
            const unsigned am = __activemask();
            const unsigned lane = threadIdx.x & 31;
            binAggregated(am, lane, key, blockCount, cellCount, &keys[i], &ranks[i]);
            if (__any_sync(am, ood) && (int)lane == __ffs(am) - 1)
                atomicOr(&hdr->status, CRB200_STATUS_OUT_OF_DOMAIN);
        }
    }

    // PB-MPM integration (pb_mpm_algorithm.h:363-408).
    template <bool Multi>
    __global__ void __launch_bounds__(128) k_pbIntegrate(const __grid_constant__ StepParams p0, SceneTable sc, float4 *__restrict__ xm,
                                                         float4 *__restrict__ vel, const unsigned char *__restrict__ mask,
                                                         float *__restrict__ F, const float *__restrict__ Cm,
                                                         unsigned stride, const ShapeRec *__restrict__ shapeTable,
                                                         SdfPtrs sdf, unsigned *status,
                                                         const unsigned long long *__restrict__ blockShapeMask)
    {
        __shared__ ShapeRec sh[Multi ? 1 : kMaxShapes];
        if (!Multi && p0.numShapes > 0)
            loadShapes(sh, shapeTable, p0.numShapes);
        __syncthreads();
        const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= (Multi ? sc.numParticles : p0.numActive) || !mask[i])
            return;
        const unsigned si = Multi ? sc.particleScene[i] : 0u;
        if (Multi && si == 0xFFFFu)
            return;
        const StepParams &p = Multi ? sc.params[si] : p0;
        const GridGeom &g = p.g;
        const ShapeRec *shp = Multi ? shapeTable + p.shapeBegin : sh;
        const float4 x4 = xm[i];
        V3 v = v3(vel[i]);
        V3 xn = v3(x4) + v * p.dt;
        xn = v3(fminf(fmaxf(xn.x, g.gmin.x), g.gmax.x), fminf(fmaxf(xn.y, g.gmin.y), g.gmax.y),
                fminf(fmaxf(xn.z, g.gmin.z), g.gmax.z));
        v = v + v3(p.gravity) * p.dt;
        if (p.numShapes > 0)
        {
            const Stencil st = stencilOf(g, v3(x4));
            int bx, by, bz;
            const unsigned blk = baseBlock(g, st, bx, by, bz);
            const bool near = st.finite && blockRegion(g, bx, by, bz).contains(xn);
            CoupleAtomic noCouple{nullptr, nullptr}; // particle push-out exchanges no momentum
            rigidContact<true>(v, x4.w, xn, shp, p.numShapes, sdf, false, noCouple,
                               near ? blockShapeMask[blk] : ~0ull);
        }
        M3 Fp, Cp, Mu;
        loadM3(F, stride, i, Fp);
        loadM3(Cm, stride, i, Cp);
#pragma unroll
        for (int e = 0; e < 9; ++e)
            Mu.m[e] = ((e % 4) == 0 ? 1.f : 0.f) + Cp.m[e] * p.dt;
        Fp = matmul(Mu, Fp);
        xm[i] = make_float4(xn.x, xn.y, xn.z, x4.w);
        vel[i] = make_float4(v.x, v.y, v.z, 0.f);
        storeM3(F, stride, i, Fp);
        if (!(isfinite(xn.x) && isfinite(xn.y) && isfinite(xn.z) && isfinite(v.x) && isfinite(v.y) && isfinite(v.z)))
            atomicOr(status, CRB200_STATUS_NAN_STATE);
    }

    // ---------------------------------------------------------------------------------------
    // computeInitialData (mls_mpm_algorithm.h:46-145): F = I, mass scatter, volume gather, then the
    // accumulation grid is cleared again.
    __global__ void k_initMass(GridGeom g0, SceneTable sc, unsigned n, const unsigned *__restrict__ idx, const float4 *__restrict__ xm,
                               float *__restrict__ F, unsigned stride, float4 *__restrict__ gridA)
    {
        const unsigned ii = blockIdx.x * blockDim.x + threadIdx.x;
        if (ii >= n)
            return;
        const unsigned p = idx[ii];
        if (sc.particleScene && sc.particleScene[p] == 0xFFFFu)
            return;
        const GridGeom g = sc.particleScene ? sc.params[sc.particleScene[p]].g : g0;
        M3 I;
#pragma unroll
        for (int e = 0; e < 9; ++e)
            I.m[e] = (e % 4) == 0 ? 1.f : 0.f;
        storeM3(F, stride, p, I);
        const float4 x4 = xm[p];
        const Stencil st = stencilOf(g, v3(x4));
        if (!st.finite)
            return;
        float w[3][3];
        weights(st.fx, w);
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 3; ++c)
                {
                    const int ni = st.b[0] + a, nj = st.b[1] + b, nk = st.b[2] + c;
                    if (!inGrid(g, ni, nj, nk))
                        continue;
                    atomicAdd(&gridA[nodeAddr(g, ni, nj, nk)].w, (w[a][0] * w[b][1] * w[c][2]) * x4.w);
                }
    }

    // Deterministic initial data: k_initMass's node masses as 64-bit fixed-point sums, which are
    // exact and so independent of the order of the atomics.  The unit is (largest particle mass) /
    // 2^50: a node sums at most a few thousand contributions of at most that mass, far below 2^63.
    __global__ void k_initMaxMass(unsigned n, const unsigned *__restrict__ idx, const float4 *__restrict__ xm,
                                  unsigned *__restrict__ maxBits)
    {
        const unsigned ii = blockIdx.x * blockDim.x + threadIdx.x;
        if (ii >= n)
            return;
        const float m = xm[idx[ii]].w;
        if (m > 0.f)
            atomicMax(maxBits, __float_as_uint(m)); // positive floats order like their bits
    }

    __global__ void k_initMassFixed(GridGeom g0, SceneTable sc, unsigned n, const unsigned *__restrict__ idx,
                                    const float4 *__restrict__ xm, float *__restrict__ F, unsigned stride,
                                    const unsigned *__restrict__ maxBits, unsigned long long *__restrict__ fixedMass)
    {
        const unsigned ii = blockIdx.x * blockDim.x + threadIdx.x;
        if (ii >= n)
            return;
        const unsigned p = idx[ii];
        if (sc.particleScene && sc.particleScene[p] == 0xFFFFu)
            return;
        const GridGeom g = sc.particleScene ? sc.params[sc.particleScene[p]].g : g0;
        M3 I;
#pragma unroll
        for (int e = 0; e < 9; ++e)
            I.m[e] = (e % 4) == 0 ? 1.f : 0.f;
        storeM3(F, stride, p, I);
        const float4 x4 = xm[p];
        const Stencil st = stencilOf(g, v3(x4));
        if (!st.finite || *maxBits == 0u)
            return;
        const double scale = 1125899906842624.0 / (double)__uint_as_float(*maxBits); // 2^50 / max mass
        float w[3][3];
        weights(st.fx, w);
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 3; ++c)
                {
                    const int ni = st.b[0] + a, nj = st.b[1] + b, nk = st.b[2] + c;
                    if (!inGrid(g, ni, nj, nk))
                        continue;
                    const float q = (w[a][0] * w[b][1] * w[c][2]) * x4.w;
                    atomicAdd(&fixedMass[nodeAddr(g, ni, nj, nk)], (unsigned long long)llrint((double)q * scale));
                }
    }

    __global__ void k_initMassFlush(unsigned numNodes, const unsigned *__restrict__ maxBits,
                                    unsigned long long *__restrict__ fixedMass, float4 *__restrict__ gridA)
    {
        const unsigned a = blockIdx.x * blockDim.x + threadIdx.x;
        if (a >= numNodes)
            return;
        const unsigned long long v = fixedMass[a];
        if (!v)
            return;
        fixedMass[a] = 0ull;
        const double unit = (double)__uint_as_float(*maxBits) / 1125899906842624.0;
        gridA[a].w += (float)((double)(long long)v * unit);
    }

    __global__ void k_initVolume(GridGeom g0, SceneTable sc, unsigned n, const unsigned *__restrict__ idx,
                                 const float4 *__restrict__ xm, const float4 *__restrict__ gridA, float *__restrict__ V0)
    {
        const unsigned ii = blockIdx.x * blockDim.x + threadIdx.x;
        if (ii >= n)
            return;
        const unsigned p = idx[ii];
        if (sc.particleScene && sc.particleScene[p] == 0xFFFFu)
            return;
        const GridGeom g = sc.particleScene ? sc.params[sc.particleScene[p]].g : g0;
        const float4 x4 = xm[p];
        const Stencil st = stencilOf(g, v3(x4));
        float dens = 0.f;
        if (st.finite)
        {
            float w[3][3];
            weights(st.fx, w);
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    for (int c = 0; c < 3; ++c)
                    {
                        const int ni = st.b[0] + a, nj = st.b[1] + b, nk = st.b[2] + c;
                        if (!inGrid(g, ni, nj, nk))
                            continue;
                        dens += (gridA[nodeAddr(g, ni, nj, nk)].w / g.cellVol) * (w[a][0] * w[b][1] * w[c][2]);
                    }
        }
        V0[p] = dens > 1e-8f ? x4.w / dens : 1e-8f;
    }

    __global__ void k_initClear(GridGeom g0, SceneTable sc, unsigned n, const unsigned *__restrict__ idx, const float4 *__restrict__ xm,
                                float4 *__restrict__ gridA)
    {
        const unsigned ii = blockIdx.x * blockDim.x + threadIdx.x;
        if (ii >= n)
            return;
        const unsigned p = idx[ii];
        if (sc.particleScene && sc.particleScene[p] == 0xFFFFu)
            return;
        const GridGeom g = sc.particleScene ? sc.params[sc.particleScene[p]].g : g0;
        const Stencil st = stencilOf(g, v3(xm[p]));
        if (!st.finite)
            return;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 3; ++c)
                {
                    const int ni = st.b[0] + a, nj = st.b[1] + b, nk = st.b[2] + c;
                    if (inGrid(g, ni, nj, nk))
                        gridA[nodeAddr(g, ni, nj, nk)] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
    }

    // Slicer cut mask of one position (checkOnDifferentSides over the 27 stencil nodes,
    // mpm_rigid_contact.h:401-478): bit a*9 + b*3 + c is set when the particle and stencil node
    // (a, b, c) lie on different sides of a slicer.
    __device__ __forceinline__ unsigned cutMaskOf(const GridGeom &g, V3 x, const Stencil &st, const ShapeRec *shp,
                                                  int numShapes, const SdfPtrs &sdf)
    {
        unsigned msk = 0;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 3; ++c)
                {
                    if (!inGrid(g, st.b[0] + a, st.b[1] + b, st.b[2] + c))
                        continue;
                    const V3 d = v3(ex::mul(ex::sub((float)a, st.fx.x), g.dx), ex::mul(ex::sub((float)b, st.fx.y), g.dx),
                                    ex::mul(ex::sub((float)c, st.fx.z), g.dx));
                    if (differentSides(x, ex::add(x, d), shp, numShapes, sdf, nullptr))
                        msk |= 1u << (a * 9 + b * 3 + c);
                }
        return msk;
    }

    // Cut masks of the current positions (bit a*9 + b*3 + c), for inspection.
    //    Multi: every particle gets a mask (zero in scenes without a slicer).
    template <bool Multi>
    __global__ void k_cutMasks(const __grid_constant__ StepParams p0, SceneTable sc, const float4 *__restrict__ xm,
                               const unsigned char *__restrict__ mask, const ShapeRec *__restrict__ shapeTable,
                               SdfPtrs sdf, unsigned *__restrict__ out)
    {
        __shared__ ShapeRec sh[Multi ? 1 : kMaxShapes];
        if (!Multi)
        {
            if (!(p0.numShapes > 0 && (sc.flags[0] & SF_SLICER)))
                return; // no slicer in the scene: masks are neither read nor kept
            loadShapes(sh, shapeTable, p0.numShapes);
            __syncthreads();
        }
        const unsigned nP = Multi ? sc.numParticles : p0.numActive;
        for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < nP; i += gridDim.x * blockDim.x)
        {
        const unsigned si = Multi ? sc.particleScene[i] : 0u;
        if (Multi && (si == 0xFFFFu || !(sc.flags[si] & SF_SLICER)))
        {
            out[i] = 0u;
            continue;
        }
        const StepParams &p = Multi ? sc.params[si] : p0;
        const GridGeom &g = p.g;
        const ShapeRec *shp = Multi ? shapeTable + p.shapeBegin : sh;
        unsigned msk = 0;
        const V3 x = v3(xm[i]);
        const Stencil st = stencilOf(g, x);
        if (st.finite && p.solverType != CRB200_SOLVER_GPU_STANDARD && mask[i])
            msk = cutMaskOf(g, x, st, shp, p.numShapes, sdf);
        out[i] = msk;
        }
    }

} // namespace crb200
#include "resident.cuh"
namespace crb200
{
    // The 3x3 SVD and the PB-MPM rotation target of a batch of matrices (column-major, 9 floats
    // each), for tests of the device arithmetic: the single-precision SVD (U, V, s) as the
    // material constraint computes it, the rotation pbRotationTarget returns, and whether that took
    // the double-precision redo.
    __global__ void k_svdBatch(unsigned n, const float *__restrict__ A, float *__restrict__ U, float *__restrict__ V,
                               float *__restrict__ S, float *__restrict__ R, unsigned *__restrict__ fp64Used,
                               unsigned *__restrict__ fp64Count)
    {
        const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n)
            return;
        M3 a;
#pragma unroll
        for (int e = 0; e < 9; ++e)
            a.m[e] = A[9ull * i + e];
        float u[9], v[9], s[3];
        svdRotations<float>(a.m, u, v, s, 5);
        const M3 r = pbRotationTarget(a, fp64Count);
#pragma unroll
        for (int e = 0; e < 9; ++e)
        {
            U[9ull * i + e] = u[e];
            V[9ull * i + e] = v[e];
            R[9ull * i + e] = r.m[e];
        }
        S[3ull * i] = s[0];
        S[3ull * i + 1] = s[1];
        S[3ull * i + 2] = s[2];
        fp64Used[i] = pbNeedsFp64(s) ? 1u : 0u;
    }

    // The adjoint's tape of one substep's sort products (read back by its reverse substep).
    __global__ void k_tapeSort(unsigned n, unsigned blocks, const unsigned *__restrict__ sortedIds,
                               const unsigned *__restrict__ cellStart, const unsigned *__restrict__ blockStart,
                               const unsigned *__restrict__ activeList, const unsigned *__restrict__ touchedList,
                               const SortHeader *__restrict__ hdr, unsigned *__restrict__ tIds, unsigned *__restrict__ tCell,
                               unsigned *__restrict__ tStart, unsigned *__restrict__ tActive,
                               unsigned *__restrict__ tTouched, SortHeader *__restrict__ tHdr)
    {
        const unsigned stepN = gridDim.x * blockDim.x, i0 = blockIdx.x * blockDim.x + threadIdx.x;
        const unsigned nSorted = min(hdr->numSorted, n), nAct = hdr->numActiveBlocks, nT = hdr->numTouchedBlocks;
        for (unsigned i = i0; i < nSorted; i += stepN)
            tIds[i] = sortedIds[i];
        for (unsigned i = i0; i < nAct * 64u; i += stepN)
        {
            const unsigned c = activeList[i >> 6] * 64u + (i & 63u);
            tCell[c] = cellStart[c];
        }
        for (unsigned i = i0; i <= blocks; i += stepN)
            tStart[i] = blockStart[i];
        for (unsigned i = i0; i < nAct; i += stepN)
            tActive[i] = activeList[i];
        for (unsigned i = i0; i < nT; i += stepN)
            tTouched[i] = touchedList[i];
        if (i0 == 0)
            *tHdr = *hdr;
    }

    // Cell keys of the most recent sort, rebuilt from its products (the per-particle key array
    // may already hold the next substep's keys, which G2P writes).
    __global__ void __launch_bounds__(64) k_sortKeysOut(const SortHeader *__restrict__ hdr,
                                                        const unsigned *__restrict__ activeList,
                                                        const unsigned *__restrict__ blockStart,
                                                        const unsigned *__restrict__ sortedIds,
                                                        const unsigned *__restrict__ cellStart,
                                                        unsigned *__restrict__ keysOut, unsigned *__restrict__ idsOut)
    {
        // keysOut: the key of every sorted particle; idsOut: each cell's ids in increasing order
        // (the canonical permutation: by key, ties by particle id)
        const unsigned nAct = hdr->numActiveBlocks;
        for (unsigned ab = blockIdx.x; ab < nAct; ab += gridDim.x)
        {
            const unsigned b = activeList[ab];
            const unsigned c = b * 64u + threadIdx.x;
            const unsigned cs = cellStart[c], ce = threadIdx.x < 63 ? cellStart[c + 1] : blockStart[b + 1];
            for (unsigned t = cs; t < ce; ++t)
            {
                const unsigned id = sortedIds[t];
                if (keysOut)
                    keysOut[id] = c;
                if (idsOut)
                {
                    // insertion into the already written, sorted prefix of this cell
                    unsigned u = t;
                    while (u > cs && idsOut[u - 1] > id)
                    {
                        idsOut[u] = idsOut[u - 1];
                        --u;
                    }
                    idsOut[u] = id;
                }
            }
        }
    }


    // ---------------------------------------------------------------------------------------
    // Host side
    static thread_local std::string g_lastError;
    static std::atomic<uint64_t> g_launches{0};

    void setLastError(const std::string &msg) { g_lastError = msg; }
    const char *lastError() { return g_lastError.c_str(); }
    void noteLaunches(uint64_t n) { g_launches.fetch_add(n); }
    uint64_t launchCount() { return g_launches.load(); }

    int cudaFail(cudaError_t e, const char *what)
    {
        if (e == cudaSuccess)
            return CRB200_OK;
        setLastError(std::string(what) + ": " + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? CRB200_ERR_OUT_OF_MEMORY : CRB200_ERR_CUDA;
    }

#define CRB_CHECK(call)                                     \
    do                                                      \
    {                                                       \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess)                              \
            return cudaFail(e_, #call);                     \
    } while (0)

#define CRB_LAUNCHED(n)                                     \
    do                                                      \
    {                                                       \
        noteLaunches(n);                                    \
        cudaError_t e_ = cudaGetLastError();                \
        if (e_ != cudaSuccess)                              \
            return cudaFail(e_, "kernel launch");           \
    } while (0)

    GridGeom makeGridGeom(float cellSize, const float mn[3], const float mx[3], unsigned blockBase)
    {
        // Node counts exactly like the reference constructor (gpu_mls_mpm_solver.cu:40-52):
        // int((max - min) / dx + 1) in single precision.
        float dims[3];
        for (int d = 0; d < 3; ++d)
        {
            volatile float size = mx[d] - mn[d];
            volatile float q = size / cellSize;
            dims[d] = q + 1.0f;
        }
        GridGeom g;
        g.gmin = make_float3(mn[0], mn[1], mn[2]);
        g.gmax = make_float3(mx[0], mx[1], mx[2]);
        g.dx = cellSize;
        g.invDx = 1 / cellSize;
        g.cellVol = cellSize * cellSize * cellSize;
        g.n = make_int3((int)dims[0], (int)dims[1], (int)dims[2]);
        g.nb = make_int3((g.n.x + 5) >> 2, (g.n.y + 5) >> 2, (g.n.z + 5) >> 2);
        g.blockBase = blockBase;
        return g;
    }

    Solver::Solver(int type, int nmax, float cellSize, const float mn[3], const float mx[3], cudaStream_t s)
        : solverType(type), numMaxParticles(nmax), stream(s)
    {
        geom = makeGridGeom(cellSize, mn, mx, 0);
        totalBlocks = (unsigned)geom.nb.x * geom.nb.y * geom.nb.z;
        numTiles = (totalBlocks + kScanTile - 1) / kScanTile;
    }

    // Scenes are laid out back to back: grids in block order (scene s owns blocks
    // [blockBase_s, blockBase_s + nb_s)), particles and shapes at the descriptor's offsets.
    Solver::Solver(int type, int nmax, const CrB200BatchSceneDesc *scenes, int n, int iters, cudaStream_t s)
        : solverType(type), numMaxParticles(nmax), stream(s)
    {
        batch.assign(scenes, scenes + n);
        iterations = iters;
        unsigned base = 0;
        for (int i = 0; i < n; ++i)
        {
            const GridGeom g = makeGridGeom(scenes[i].cellSize, scenes[i].gridMin, scenes[i].gridMax, base);
            batchGeom.push_back(g);
            base += (unsigned)g.nb.x * g.nb.y * g.nb.z;
        }
        geom = batchGeom[0];
        dt = scenes[0].dt;
        gravity = make_float3(scenes[0].gravity[0], scenes[0].gravity[1], scenes[0].gravity[2]);
        contactModel = scenes[0].contactModel;
        numActive = totalParticles();
        numShapes = totalShapes();
        totalBlocks = base;
        numTiles = (totalBlocks + kScanTile - 1) / kScanTile;
    }

    unsigned Solver::totalParticles() const
    {
        if (!isBatch())
            return numActive;
        unsigned n = 0;
        for (const auto &d : batch)
            n = std::max(n, (unsigned)(d.particleOffset + d.numParticles));
        return n;
    }

    int Solver::totalShapes() const
    {
        if (!isBatch())
            return numShapes;
        int n = 0;
        for (const auto &d : batch)
            n = std::max(n, d.shapeOffset + d.numShapes);
        return n;
    }

    std::vector<StepParams> Solver::allParams() const
    {
        std::vector<StepParams> out;
        if (!isBatch())
        {
            out.push_back(params());
            return out;
        }
        for (size_t i = 0; i < batch.size(); ++i)
        {
            const CrB200BatchSceneDesc &d = batch[i];
            StepParams p;
            p.g = batchGeom[i];
            p.dt = d.dt;
            p.gravity = make_float3(d.gravity[0], d.gravity[1], d.gravity[2]);
            p.cutoff = solverType == CRB200_SOLVER_GPU_PB ? 1e-8f : 1e-4f;
            p.contactModel = d.contactModel;
            p.solverType = solverType;
            p.numActive = (unsigned)d.numParticles;
            p.numShapes = d.numShapes;
            p.particleBegin = (unsigned)d.particleOffset;
            p.shapeBegin = d.shapeOffset;
            p.pad = 0;
            out.push_back(p);
        }
        return out;
    }

    // Scene parameters live on the device for batches; setters re-upload them between substeps.
    int Solver::uploadParams()
    {
        if (!isBatch() || !dParams)
            return CRB200_OK;
        const std::vector<StepParams> ps = allParams();
        CRB_CHECK(cudaStreamSynchronize(stream));
        CRB_CHECK(cudaMemcpy(dParams, ps.data(), ps.size() * sizeof(StepParams), cudaMemcpyHostToDevice));
        return CRB200_OK;
    }

    SceneTable Solver::sceneTable() const
    {
        SceneTable t;
        t.params = dParams;
        t.particleScene = dParticleScene;
        t.flags = isBatch() ? dSceneFlags : &header->shapeFlags;
        t.numScenes = numScenes();
        t.numParticles = totalParticles();
        return t;
    }

    Solver::~Solver()
    {
        if (graph)
            cudaGraphExecDestroy(graph);
        if (graphLean)
            cudaGraphExecDestroy(graphLean);
        if (graphSingle)
            cudaGraphExecDestroy(graphSingle);
        for (cudaEvent_t e : phaseEv)
            if (e)
                cudaEventDestroy(e);
        for (cudaGraphExec_t &gx : resGraph)
            if (gx)
                cudaGraphExecDestroy(gx);
        void *bufs[] = {F, Cm, V0, gridA, gridV, gridF, keys, ranks, sortedIds, cellCount, blockCount, blockStart,
                        activeList, touchedList, tileSums, cutMasks, header, shapeTable, blockFlags, records, cellStart,
                        dParams, dParticleScene, dSceneFlags, blockShapeMask, detPartials, detMask,
                        detTiles, detTilesF, detFixedMass, res.x, res.v, res.V0, res.F, res.C, const_cast<float4 *>(res.mat),
                        const_cast<unsigned *>(res.id), res.cut, resSlotOf, resX2, resV02, resMat2, resF2, resC2, resId2,
                        touchedFlag, onesMask, iotaIds};
        for (void *b : bufs)
            if (b)
                cudaFree(b);
        releaseAdjoint();
        if (copiedEvent)
            cudaEventSynchronize(copiedEvent);
        for (cudaEvent_t e : {forkEvent, stagedEvent, copiedEvent})
            if (e)
                cudaEventDestroy(e);
        if (copyStream)
            cudaStreamDestroy(copyStream);
        if (stageX)
            cudaFree(stageX);
        if (stageV)
            cudaFree(stageV);
        if (joinEvent)
            cudaEventDestroy(joinEvent);
        if (sideStream)
            cudaStreamDestroy(sideStream);
    }

    // 0: atomics; 1: coupling reduced in a fixed order; 2: also the P2G grid from block tiles.
    // The substeps an adjoint backward pass replays follow the option too, so that they reproduce
    // a deterministic recording bit for bit (their coupling goes to scratch either way).
    int Solver::detLevel(bool recomputing) const
    {
        (void)recomputing;
        if (isBatch())
            return (detP2G && detTiles) ? 2 : 0; // a batch has no fixed-order coupling
        if (!detPartials)
            return 0;
        if (detP2G && detTiles)
            return 2;
        return detCoupling ? 1 : 0;
    }

    // Deterministic substeps: tiles of every grid block (216 float4; twice for the standard
    // solver's force pass), written whole by the accumulation of each active block.
    int Solver::setDeterministic(bool on)
    {
        if (!isBatch())
            if (int rc = setDeterministicCoupling(on))
                return rc;
        if (on && !detTiles)
        {
            const size_t bytes = (size_t)totalBlocks * kTileNodes * sizeof(float4);
            CRB_CHECK(cudaMalloc(&detTiles, bytes));
            if (solverType == CRB200_SOLVER_GPU_STANDARD)
                CRB_CHECK(cudaMalloc(&detTilesF, bytes));
            // fixed-point node masses of the initial data, plus one word for the largest particle mass
            const size_t fbytes = ((size_t)totalBlocks * 64u + 1u) * sizeof(unsigned long long);
            CRB_CHECK(cudaMalloc(&detFixedMass, fbytes));
            CRB_CHECK(cudaMemset(detFixedMass, 0, fbytes));
        }
        detP2G = on;
        return CRB200_OK;
    }

    // Deterministic coupling: the block partial buffer (zeroed; the reduction keeps it zeroed).
    int Solver::setDeterministicCoupling(bool on)
    {
        if (on && isBatch())
        {
            setLastError("deterministic coupling: not available on batch solvers");
            return CRB200_ERR_UNSUPPORTED;
        }
        if (on && !detPartials)
        {
            const size_t bytes = (size_t)totalBlocks * kDetSlots * 2 * sizeof(float4);
            const size_t maskBytes = ((size_t)(totalBlocks + 31) / 32 + 1) * sizeof(unsigned); // + the "any" word
            CRB_CHECK(cudaMalloc(&detPartials, bytes));
            CRB_CHECK(cudaMemset(detPartials, 0, bytes));
            CRB_CHECK(cudaMalloc(&detMask, maskBytes));
            CRB_CHECK(cudaMemset(detMask, 0, maskBytes));
        }
        detCoupling = on;
        return CRB200_OK;
    }

    StepParams Solver::params() const
    {
        StepParams p;
        p.g = geom;
        p.dt = dt;
        p.gravity = gravity;
        p.cutoff = solverType == CRB200_SOLVER_GPU_PB ? 1e-8f : 1e-4f;
        p.contactModel = contactModel;
        p.solverType = solverType;
        p.numActive = numActive;
        p.numShapes = numShapes;
        p.particleBegin = 0;
        p.shapeBegin = 0;
        p.pad = 0;
        return p;
    }

    int Solver::initialize()
    {
        if (!positionMass || !velocity)
        {
            setLastError("initialize: particle data not bound");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        const size_t n = (size_t)numMaxParticles;
        const size_t nodes = (size_t)totalBlocks * 64;
        CRB_CHECK(cudaMalloc(&F, 9 * n * sizeof(float)));
        CRB_CHECK(cudaMalloc(&Cm, 9 * n * sizeof(float)));
        CRB_CHECK(cudaMalloc(&V0, n * sizeof(float)));
        CRB_CHECK(cudaMalloc(&gridA, nodes * sizeof(float4)));
        CRB_CHECK(cudaMalloc(&gridV, nodes * sizeof(float4)));
        if (solverType == CRB200_SOLVER_GPU_STANDARD)
            CRB_CHECK(cudaMalloc(&gridF, nodes * sizeof(float4)));
        CRB_CHECK(cudaMalloc(&keys, n * sizeof(unsigned)));
        CRB_CHECK(cudaMalloc(&ranks, n * sizeof(unsigned)));
        CRB_CHECK(cudaMalloc(&sortedIds, n * sizeof(unsigned)));
        CRB_CHECK(cudaMalloc(&cellCount, (size_t)totalBlocks * 64 * sizeof(unsigned)));
        CRB_CHECK(cudaMalloc(&cellStart, (size_t)totalBlocks * 64 * sizeof(unsigned)));
        CRB_CHECK(cudaMemsetAsync(cellCount, 0, (size_t)totalBlocks * 64 * sizeof(unsigned), stream));
        CRB_CHECK(cudaMalloc(&blockCount, (totalBlocks + 1) * sizeof(unsigned)));
        CRB_CHECK(cudaMalloc(&blockStart, (totalBlocks + 1) * sizeof(unsigned)));
        CRB_CHECK(cudaMalloc(&activeList, totalBlocks * sizeof(unsigned)));
        CRB_CHECK(cudaMalloc(&touchedList, totalBlocks * sizeof(unsigned)));
        CRB_CHECK(cudaMalloc(&tileSums, numTiles * sizeof(uint3)));
        CRB_CHECK(cudaMalloc(&blockFlags, totalBlocks));
        CRB_CHECK(cudaMalloc(&blockShapeMask, totalBlocks * sizeof(unsigned long long)));
        CRB_CHECK(cudaMalloc(&header, sizeof(SortHeader)));
        const int shapeSlots = isBatch() ? std::max(totalShapes(), 1) : kMaxShapes;
        CRB_CHECK(cudaMalloc(&shapeTable, shapeSlots * sizeof(ShapeRec)));
        if (isBatch())
        {
            std::vector<unsigned short> owner(n, 0xFFFF);
            for (size_t i = 0; i < batch.size(); ++i)
                for (int q = 0; q < batch[i].numParticles; ++q)
                    owner[batch[i].particleOffset + q] = (unsigned short)i;
            CRB_CHECK(cudaMalloc(&dParams, batch.size() * sizeof(StepParams)));
            CRB_CHECK(cudaMalloc(&dParticleScene, n * sizeof(unsigned short)));
            CRB_CHECK(cudaMalloc(&dSceneFlags, batch.size() * sizeof(unsigned)));
            CRB_CHECK(cudaMemcpy(dParticleScene, owner.data(), n * sizeof(unsigned short), cudaMemcpyHostToDevice));
            CRB_CHECK(cudaMemset(dSceneFlags, 0, batch.size() * sizeof(unsigned)));
            const std::vector<StepParams> ps = allParams();
            CRB_CHECK(cudaMemcpy(dParams, ps.data(), ps.size() * sizeof(StepParams), cudaMemcpyHostToDevice));
        }
        CRB_CHECK(cudaMalloc(&cutMasks, n * sizeof(unsigned)));
        CRB_CHECK(cudaMalloc(&records, n * 4 * sizeof(float4)));
        CRB_CHECK(cudaMemsetAsync(F, 0, 9 * n * sizeof(float), stream));
        CRB_CHECK(cudaMemsetAsync(Cm, 0, 9 * n * sizeof(float), stream));
        CRB_CHECK(cudaMemsetAsync(V0, 0, n * sizeof(float), stream));
        CRB_CHECK(cudaMemsetAsync(gridA, 0, nodes * sizeof(float4), stream));
        CRB_CHECK(cudaMemsetAsync(gridV, 0, nodes * sizeof(float4), stream));
        if (gridF)
            CRB_CHECK(cudaMemsetAsync(gridF, 0, nodes * sizeof(float4), stream));
        CRB_CHECK(cudaMemsetAsync(blockCount, 0, (totalBlocks + 1) * sizeof(unsigned), stream));
        CRB_CHECK(cudaMemsetAsync(header, 0, sizeof(SortHeader), stream));
        CRB_CHECK(cudaMemsetAsync(keys, 0xff, n * sizeof(unsigned), stream));
        int dev = 0, sms = 0, perSm = 0;
        CRB_CHECK(cudaGetDevice(&dev));
        CRB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        CRB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_accumulate<0, false>, 64, 0));
        p2gCtas = sms * (perSm > 0 ? perSm : 1);
        sortCtas = sms * 4;  // 64-thread CTAs of the on-request sort-state kernel
        cellCtas = sms * 4;  // 256-thread CTAs of k_cellStarts (one warp per active block)
        updCtas = sms * 8;
        CRB_CHECK(cudaStreamCreateWithFlags(&sideStream, cudaStreamNonBlocking));
        CRB_CHECK(cudaEventCreateWithFlags(&forkEvent, cudaEventDisableTiming));
        CRB_CHECK(cudaEventCreateWithFlags(&joinEvent, cudaEventDisableTiming));
        strideCtas = sms * 16; // grid-stride kernels of 128 threads: a full SM each
        initialized = true;
        configVersion++;
        return CRB200_OK;
    }

    void Solver::gatherShapes(cudaStream_t s)
    {
        k_gatherShapes<<<numScenes(), 64, 0, s>>>(params(), sceneTable(), shapeIds, shapes, geometries, shapeTable);
    }

    int Solver::sortParticles(const StepParams &p, bool ignoreMask)
    {
        const SceneTable sc = sceneTable();
        const unsigned n = sc.numParticles;
        const unsigned pg = (n + 127) / 128;
        if (n > 0)
        {
            if (isBatch())
                k_bin<true><<<pg, 128, 0, stream>>>(p, sc, ignoreMask, positionMass, activeMask, keys, ranks, blockCount,
                                                    cellCount, header);
            else
                k_bin<false><<<pg, 128, 0, stream>>>(p, sc, ignoreMask, positionMass, activeMask, keys, ranks, blockCount,
                                                     cellCount, header);
            CRB_LAUNCHED(1);
        }
        unsigned char *flags = blockFlags;
        k_scanReduce<<<numTiles, kScanThreads, 0, stream>>>(p, sc, totalBlocks, blockCount, flags,
                                                            reinterpret_cast<uint3 *>(tileSums), header);
        k_scanTiles<<<1, 1024, 0, stream>>>(reinterpret_cast<uint3 *>(tileSums), numTiles, header,
                                            (unsigned)numMaxParticles);
        k_scanWrite<<<numTiles, kScanThreads, 0, stream>>>(totalBlocks, reinterpret_cast<const uint3 *>(tileSums),
                                                           blockCount, flags, blockStart, activeList, touchedList,
                                                           header);
        CRB_LAUNCHED(3);
        if (n > 0)
        {
            k_cellStarts<<<cellCtas, 256, 0, stream>>>(header, activeList, blockStart, cellCount, cellStart);
            k_scatter<<<pg, 128, 0, stream>>>(n, keys, ranks, cellStart, sortedIds, (unsigned)numMaxParticles, header);
            CRB_LAUNCHED(1);
        }
        return CRB200_OK;
    }
} // namespace crb200

namespace crb200
{
    int Solver::launchStep()
    {
        if (isBatch())
            return launchStepT<true>(false);
        return launchStepT<false>(false);
    }

    // recompute: a forward substep up to the grid update only (the adjoint's replay of a segment's
    // last input state); coupling forces go to scratch.  With a tape slot active (tapeActive) the
    // grid update also writes the P2G grid and the grid velocities to that slot, and the sort
    // products are copied there; otherwise recompute keeps the P2G grid in gridA.
    template <bool Multi>
    int Solver::launchStepT(bool recompute)
    {
        if (!Multi && numShapes > kMaxShapes)
        {
            setLastError("step: more than 64 shapes in one scene");
            return CRB200_ERR_CAPACITY;
        }
        if (numShapes > 0 && (!shapeIds || !shapes.type || !geometries.type))
        {
            setLastError("step: shapes are enabled but shape ids / shape data / geometry data are not bound");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        if (numActive > 0 && (!matParams || !matType || !activeMask))
        {
            setLastError("step: particle materials or active mask not bound");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        const StepParams p = params();
        const SceneTable sc = sceneTable();
        const unsigned nPart = sc.numParticles;
        markPhase(0);
        const bool isStd = solverType == CRB200_SOLVER_GPU_STANDARD;
        // The shape gather and the slicer cut masks depend on the shapes and the positions only:
        // they run on a side stream beside the sort chain and join before P2G (graph branches
        // when captured).
        const bool fork = numShapes > 0 && sideStream != nullptr && stream != nullptr && !phaseTiming;
        cudaStream_t shapeStream = stream;
        if (fork)
        {
            CRB_CHECK(cudaEventRecord(forkEvent, stream));
            CRB_CHECK(cudaStreamWaitEvent(sideStream, forkEvent, 0));
            shapeStream = sideStream;
        }
        if (numShapes > 0)
        {
            gatherShapes(shapeStream);
            CRB_LAUNCHED(1);
        }
        const SdfPtrs sp{reinterpret_cast<const int4 *>(sdf.dimension), reinterpret_cast<const float4 *>(sdf.lowerBoundCellSize),
                         reinterpret_cast<const float4 *>(sdf.gradientSignedDistance)};
        float4 *cf = reinterpret_cast<float4 *>(shapes.force), *ct = reinterpret_cast<float4 *>(shapes.torque);
        const unsigned stride = (unsigned)numMaxParticles;
        const unsigned pg = (nPart + 127) / 128;
        // Slicer cut masks of this substep's positions (positions do not change across PB-MPM
        // iterations, so one evaluation serves every iteration of the step).
        if (numShapes > 0 && !isStd && pg)
        {
            k_cutMasks<Multi><<<std::min(pg, (unsigned)strideCtas), 128, 0, shapeStream>>>(p, sc, positionMass, activeMask,
                                                                                          shapeTable, sp, cutMasks);
            CRB_LAUNCHED(1);
        }
        if (fork)
            CRB_CHECK(cudaEventRecord(joinEvent, sideStream));
        int r = sortParticles(p, isStd);
        if (r != CRB200_OK)
            return r;
        if (nPart > 0 && detLevel(recompute || adjReplay) == 2)
        {
            k_cellOrder<<<cellCtas * 4, 64, 0, stream>>>(header, activeList, blockStart, cellStart, sortedIds);
            CRB_LAUNCHED(1);
        }
        if (fork)
            CRB_CHECK(cudaStreamWaitEvent(stream, joinEvent, 0));
        markPhase(1);
        auto p2g = [&](auto mode) -> int {
            constexpr int M = decltype(mode)::value;
            if (!pg)
                return CRB200_OK;
            k_record<M, Multi><<<std::min(pg, (unsigned)strideCtas), 128, 0, stream>>>(p, sc, header, sortedIds, positionMass, velocity, matParams, matType,
                                                        F, Cm, V0, stride, cutMasks, records, gridA, gridF,
                                                        &header->fp64Fallbacks);
            bool tiled = false;
            if (detLevel(recompute || adjReplay) == 2)
            {
                k_accumulate<M, Multi, true><<<p2gCtas, 64, 0, stream>>>(p, sc, header, activeList, blockStart,
                                                                       sortedIds, cellStart, records, cutMasks,
                                                                       gridA, gridF, detTiles, detTilesF);
                tiled = true;
            }
            if (!tiled)
                k_accumulate<M, Multi><<<p2gCtas, 64, 0, stream>>>(p, sc, header, activeList, blockStart, sortedIds,
                                                                    cellStart, records, cutMasks, gridA, gridF);
            CRB_LAUNCHED(2);
            return CRB200_OK;
        };
        auto update = [&]() -> int {
            const int det = detLevel(recompute || adjReplay);
            auto upd = [&](auto detTag) {
                constexpr int D = decltype(detTag)::value;
                k_gridUpdate<Multi, D><<<updCtas, 256, 0, stream>>>(
                    p, sc, header, touchedList, shapeTable, sp, gridA, gridF, gridV, (recompute || adjReplay) ? adjForce : cf,
                    (recompute || adjReplay) ? adjTorque : ct, !recompute || tapeActive >= 0, blockShapeMask,
                    tapeActive >= 0 ? tapeSlot(tapeActive).gridA : nullptr,
                    tapeActive >= 0 ? tapeSlot(tapeActive).gridV : nullptr, D ? detPartials : nullptr,
                    D ? detMask : nullptr, (totalBlocks + 31) / 32, D == 2 ? detTiles : nullptr, D == 2 ? detTilesF : nullptr,
                    blockFlags);
            };
            if constexpr (!Multi)
                if (det != 0)
                {
                    if (det == 2)
                        upd(std::integral_constant<int, 2>{});
                    else
                        upd(std::integral_constant<int, 1>{});
                    k_coupleReduce<<<1, 256, 0, stream>>>((totalBlocks + 31) / 32, detMask, detPartials, shapeTable,
                                                          numShapes, (recompute || adjReplay) ? adjForce : cf,
                                                          (recompute || adjReplay) ? adjTorque : ct);
                    CRB_LAUNCHED(2);
                }
            if constexpr (Multi)
                if (det == 2) // the tiles in a fixed order; the coupling of dynamic shapes stays atomic
                {
                    upd(std::integral_constant<int, 2>{});
                    CRB_LAUNCHED(1);
                }
            if (det == 0)
            {
                upd(std::integral_constant<int, 0>{});
                CRB_LAUNCHED(1);
            }
            if (tapeActive >= 0)
            {
                const TapeSlot ts = tapeSlot(tapeActive);
                k_tapeSort<<<strideCtas, 256, 0, stream>>>(totalParticles(), totalBlocks, sortedIds, cellStart, blockStart,
                                                          activeList, touchedList, header, ts.sortedIds, ts.cellStart,
                                                          ts.blockStart, ts.activeList, ts.touchedList, ts.hdr);
                CRB_LAUNCHED(1);
            }
            return CRB200_OK;
        };
        // pbRecords: PB-MPM iterations but the last build the next iteration's records in G2P
        auto g2p = [&](auto mode, bool pbRecords = false) -> int {
            constexpr int M = decltype(mode)::value;
            if (!pg)
                return CRB200_OK;
            const unsigned char *g2pMask = (M == 2 && stdGpuSemantics && onesMask) ? onesMask : activeMask;
            k_g2p<M, Multi><<<pg, 128, 0, stream>>>(p, sc, positionMass, velocity, g2pMask, F, Cm, stride, shapeTable,
                                                    sp, gridV, cutMasks, &header->status, matParams, matType, V0,
                                                    (M == 0 || (M == 1 && pbRecords)) ? records : nullptr, gridA, header, keys, ranks,
                                                    blockCount, cellCount, blockShapeMask,
                                                    outX ? outX : positionMass, outX ? outV : velocity,
                                                    outX ? outF : F, outX ? outC : Cm,
                                                    M == 0 && !Multi && leanG2P && outX == nullptr);
            CRB_LAUNCHED(1);
            return CRB200_OK;
        };
        using M0 = std::integral_constant<int, 0>;
        using M1 = std::integral_constant<int, 1>;
        using M2 = std::integral_constant<int, 2>;
        if (solverType == CRB200_SOLVER_GPU_MLS)
        {
            if ((r = p2g(M0{})) != CRB200_OK) return r;
            markPhase(2);
            if ((r = update()) != CRB200_OK) return r;
            if (recompute)
                return CRB200_OK;
            markPhase(3);
            if ((r = g2p(M0{})) != CRB200_OK) return r;
        }
        else if (solverType == CRB200_SOLVER_GPU_PB)
        {
            for (int it = 0; it < iterations; ++it)
            {
                if ((r = p2g(M1{})) != CRB200_OK) return r;
                if (it == 0) markPhase(2);
                if ((r = update()) != CRB200_OK) return r;
                if (it == 0) markPhase(3);
                if ((r = g2p(M1{}, it + 1 < iterations)) != CRB200_OK) return r;
            }
            if (pg)
            {
                k_pbIntegrate<Multi><<<pg, 128, 0, stream>>>(p, sc, positionMass, velocity, activeMask, F, Cm, stride,
                                                             shapeTable, sp, &header->status, blockShapeMask);
                CRB_LAUNCHED(1);
            }
        }
        else
        {
            if ((r = p2g(M2{})) != CRB200_OK) return r;
            markPhase(2);
            if ((r = update()) != CRB200_OK) return r;
            markPhase(3);
            if ((r = g2p(M2{})) != CRB200_OK) return r;
        }
        markPhase(4);
        if (phaseTiming)
            return collectPhaseTimes();
        return CRB200_OK;
    }

    // Phase events (PB-MPM folds all iterations' P2G / update / G2P into phases 1-3 by recording the
    // boundaries of the first iteration only and scaling; see collectPhaseTimes).
    int Solver::markPhase(int k)
    {
        if (!phaseTiming)
            return CRB200_OK;
        if (!phaseEv[k])
            CRB_CHECK(cudaEventCreate(&phaseEv[k]));
        CRB_CHECK(cudaEventRecord(phaseEv[k], stream));
        return CRB200_OK;
    }

    int Solver::collectPhaseTimes()
    {
        CRB_CHECK(cudaEventSynchronize(phaseEv[4]));
        for (int k = 0; k < 4; ++k)
        {
            float ms = 0.f;
            CRB_CHECK(cudaEventElapsedTime(&ms, phaseEv[k], phaseEv[k + 1]));
            phaseMs[k] += ms;
        }
        phaseSteps++;
        return CRB200_OK;
    }

    int Solver::advance(float dtFrame, float4 *hostX, float4 *hostV, int *outSubsteps)
    {
        for (const auto &d : batch)
            if (d.dt != dt)
            {
                setLastError("advance: the scenes of this batch have different substep sizes");
                return CRB200_ERR_UNSUPPORTED;
            }
        // scene_impl.cpp:313-317: float time accumulation decides the substep count
        float t = 0.f;
        int n = 0;
        while (t < dtFrame)
        {
            t += dt;
            ++n;
        }
        int r = stepMany(n);
        if (r != CRB200_OK)
            return r;
        const unsigned nPart = totalParticles();
        if (hostX && nPart)
            CRB_CHECK(cudaMemcpyAsync(hostX, positionMass, nPart * sizeof(float4), cudaMemcpyDeviceToHost, stream));
        if (hostV && nPart)
            CRB_CHECK(cudaMemcpyAsync(hostV, velocity, nPart * sizeof(float4), cudaMemcpyDeviceToHost, stream));
        CRB_CHECK(cudaStreamSynchronize(stream));
        if (outSubsteps)
            *outSubsteps = n;
        return CRB200_OK;
    }

    // Asynchronous variant of advance: the substeps, a device-side snapshot of x and v, and their
    // copy to the host on a separate copy stream are enqueued, and the call returns; the next
    // frame's substeps overlap this frame's readback.  fetchResults waits for both.
    int Solver::advanceAsync(float dtFrame, float4 *hostX, float4 *hostV, int *outSubsteps)
    {
        for (const auto &d : batch)
            if (d.dt != dt)
            {
                setLastError("advance: the scenes of this batch have different substep sizes");
                return CRB200_ERR_UNSUPPORTED;
            }
        if (stream == nullptr)
        {
            setLastError("advanceAsync: needs a non-default solver stream");
            return CRB200_ERR_UNSUPPORTED;
        }
        float t = 0.f;
        int n = 0;
        while (t < dtFrame)
        {
            t += dt;
            ++n;
        }
        int r = stepMany(n);
        if (r != CRB200_OK)
            return r;
        const unsigned nPart = totalParticles();
        if ((hostX || hostV) && nPart)
        {
            if (!copyStream)
            {
                CRB_CHECK(cudaStreamCreateWithFlags(&copyStream, cudaStreamNonBlocking));
                CRB_CHECK(cudaEventCreateWithFlags(&stagedEvent, cudaEventDisableTiming));
                CRB_CHECK(cudaEventCreateWithFlags(&copiedEvent, cudaEventDisableTiming));
                CRB_CHECK(cudaMalloc(&stageX, (size_t)numMaxParticles * sizeof(float4)));
                CRB_CHECK(cudaMalloc(&stageV, (size_t)numMaxParticles * sizeof(float4)));
                CRB_CHECK(cudaEventRecord(copiedEvent, copyStream));
            }
            // the previous frame's host copy must be done with the staging buffers
            CRB_CHECK(cudaStreamWaitEvent(stream, copiedEvent, 0));
            if (hostX)
                CRB_CHECK(cudaMemcpyAsync(stageX, positionMass, nPart * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
            if (hostV)
                CRB_CHECK(cudaMemcpyAsync(stageV, velocity, nPart * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
            CRB_CHECK(cudaEventRecord(stagedEvent, stream));
            CRB_CHECK(cudaStreamWaitEvent(copyStream, stagedEvent, 0));
            if (hostX)
                CRB_CHECK(cudaMemcpyAsync(hostX, stageX, nPart * sizeof(float4), cudaMemcpyDeviceToHost, copyStream));
            if (hostV)
                CRB_CHECK(cudaMemcpyAsync(hostV, stageV, nPart * sizeof(float4), cudaMemcpyDeviceToHost, copyStream));
            CRB_CHECK(cudaEventRecord(copiedEvent, copyStream));
        }
        if (outSubsteps)
            *outSubsteps = n;
        return CRB200_OK;
    }

    int Solver::step()
    {
        if (!initialized)
        {
            setLastError("step: solver not initialized");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        if (residentUsable())
            return residentStep(1);
        int r = residentRetire(); // back to the particle-id order if the resident path ran before
        if (r != CRB200_OK)
            return r;
        if (stream == nullptr || phaseTiming)
        {
            r = invalidateRecords();
            return r != CRB200_OK ? r : launchStep();
        }
        // A scene steps one substep per call (scene_impl.cpp:314-317): the record invalidation and
        // the substep are replayed from one captured graph, one launch on the host instead of a
        // dozen.
        if (graphSingle == nullptr || graphSingleVersion != configVersion)
        {
            if (graphSingle)
            {
                cudaGraphExecDestroy(graphSingle);
                graphSingle = nullptr;
            }
            const uint64_t before = launchCount();
            CRB_CHECK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            r = invalidateRecords();
            if (r == CRB200_OK)
                r = launchStep();
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(stream, &g);
            const uint64_t captured = launchCount() - before;
            noteLaunches((uint64_t)0 - captured); // captured, not yet executed
            if (r != CRB200_OK)
            {
                if (g)
                    cudaGraphDestroy(g);
                return r;
            }
            if (e != cudaSuccess)
                return cudaFail(e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&graphSingle, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess)
                return cudaFail(e, "cudaGraphInstantiate");
            graphSingleKernels = (int)captured;
            graphSingleVersion = configVersion;
        }
        CRB_CHECK(cudaGraphLaunch(graphSingle, stream));
        noteLaunches((uint64_t)graphSingleKernels);
        return CRB200_OK;
    }

    // Bins and P2G records written by G2P hold for the next substep of the same call only: the
    // caller may change particle buffers, materials or parameters between calls.  The block counts
    // the last G2P of a call accumulated for a substep that did not follow are cleared with the
    // flag, so that k_bin starts from zero counts.
    int Solver::invalidateRecords()
    {
        CRB_CHECK(cudaMemsetAsync(&header->recordsValid, 0, 3 * sizeof(unsigned), stream)); // + pbRecordsValid, sortSkip
        CRB_CHECK(cudaMemsetAsync(blockCount, 0, (totalBlocks + 1) * sizeof(unsigned), stream));
        CRB_CHECK(cudaMemsetAsync(cellCount, 0, (size_t)totalBlocks * 64 * sizeof(unsigned), stream));
        return CRB200_OK;
    }

    int Solver::stepMany(int n)
    {
        if (!initialized)
        {
            setLastError("stepMany: solver not initialized");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        if (n <= 0)
            return CRB200_OK;
        if (residentUsable())
            return residentStep(n);
        int rv = residentRetire(); // back to the particle-id order if the resident path ran before
        if (rv == CRB200_OK)
            rv = invalidateRecords();
        if (rv != CRB200_OK)
            return rv;
        if (stream == nullptr || n < 2 || phaseTiming)
        {
            for (int i = 0; i < n; ++i)
            {
                int r = launchStep();
                if (r != CRB200_OK)
                    return r;
            }
            return CRB200_OK;
        }
        if (graph == nullptr || graphVersion != configVersion)
        {
            for (cudaGraphExec_t *gx : {&graph, &graphLean})
                if (*gx)
                {
                    cudaGraphExecDestroy(*gx);
                    *gx = nullptr;
                }
            // the full substep, and (single-scene MLS) the lean one for all but a call's last
            const bool withLean = !isBatch() && solverType == CRB200_SOLVER_GPU_MLS;
            for (int k = 0; k < (withLean ? 2 : 1); ++k)
            {
                const uint64_t before = launchCount();
                leanG2P = k == 1;
                CRB_CHECK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
                int r = launchStep();
                cudaGraph_t g = nullptr;
                cudaError_t e = cudaStreamEndCapture(stream, &g);
                leanG2P = false;
                const uint64_t captured = launchCount() - before;
                noteLaunches((uint64_t)0 - captured); // captured, not yet executed
                if (r != CRB200_OK)
                {
                    if (g)
                        cudaGraphDestroy(g);
                    return r;
                }
                if (e != cudaSuccess)
                    return cudaFail(e, "cudaStreamEndCapture");
                e = cudaGraphInstantiate(k == 1 ? &graphLean : &graph, g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess)
                    return cudaFail(e, "cudaGraphInstantiate");
                graphKernels = (int)captured;
            }
            graphVersion = configVersion;
        }
        for (int i = 0; i < n - 1; ++i)
            CRB_CHECK(cudaGraphLaunch(graphLean ? graphLean : graph, stream));
        CRB_CHECK(cudaGraphLaunch(graph, stream));
        noteLaunches((uint64_t)graphKernels * (uint64_t)n);
        return CRB200_OK;
    }

    __global__ void k_iota(unsigned n, unsigned *__restrict__ out)
    {
        for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            out[i] = i;
    }

    // The reference's GPU standard-MPM solver reads the active mask in P2G only and ignores the
    // index list of computeInitialData, initialising particles 0..n-1
    // (gpu_standard_mpm_solver.cu:210-212, 280-282, 357-359); its CPU solver honours both.  The
    // engine follows the CPU solver unless this is on.
    int Solver::setStdGpuSemantics(bool on)
    {
        if (on && !onesMask)
        {
            const size_t n = (size_t)numMaxParticles;
            CRB_CHECK(cudaMalloc(&onesMask, n));
            CRB_CHECK(cudaMalloc(&iotaIds, n * sizeof(unsigned)));
            CRB_CHECK(cudaMemsetAsync(onesMask, 1, n, stream));
            // (may run before initialize(), so the grid is sized here)
            k_iota<<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0, stream>>>((unsigned)n, iotaIds);
            CRB_LAUNCHED(1);
        }
        if (stdGpuSemantics != on)
            configVersion++;
        stdGpuSemantics = on;
        return CRB200_OK;
    }

    int Solver::computeInitialData(unsigned n, const unsigned *indices)
    {
        if (!initialized)
        {
            setLastError("computeInitialData: solver not initialized");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        if (n == 0)
            return CRB200_OK;
        if (!indices)
        {
            setLastError("computeInitialData: null index list");
            return CRB200_ERR_INVALID_ARGUMENT;
        }
        // F = I and V0 of the listed particles go to the particle-id planes: the resident state is
        // synced first and re-sorted from the planes at the next resident call
        if (int r = residentRetire())
            return r;
        if (stdGpuSemantics && solverType == CRB200_SOLVER_GPU_STANDARD && !isBatch())
        {
            if (n > (unsigned)numMaxParticles)
            {
                setLastError("computeInitialData: more particles than numMaxParticles");
                return CRB200_ERR_INVALID_ARGUMENT;
            }
            indices = iotaIds; // particles 0..n-1, whatever the list
        }
        const unsigned g = (n + 127) / 128;
        const SceneTable sc = sceneTable();
        if (detP2G && detFixedMass)
        {
            unsigned *maxBits = reinterpret_cast<unsigned *>(detFixedMass + (size_t)totalBlocks * 64u);
            CRB_CHECK(cudaMemsetAsync(maxBits, 0, sizeof(unsigned), stream));
            k_initMaxMass<<<g, 128, 0, stream>>>(n, indices, positionMass, maxBits);
            k_initMassFixed<<<g, 128, 0, stream>>>(geom, sc, n, indices, positionMass, F, (unsigned)numMaxParticles,
                                                   maxBits, detFixedMass);
            const unsigned nodes = totalBlocks * 64u;
            k_initMassFlush<<<(nodes + 255) / 256, 256, 0, stream>>>(nodes, maxBits, detFixedMass, gridA);
            CRB_LAUNCHED(3);
        }
        else
        {
            k_initMass<<<g, 128, 0, stream>>>(geom, sc, n, indices, positionMass, F, (unsigned)numMaxParticles, gridA);
            CRB_LAUNCHED(1);
        }
        k_initVolume<<<g, 128, 0, stream>>>(geom, sc, n, indices, positionMass, gridA, V0);
        k_initClear<<<g, 128, 0, stream>>>(geom, sc, n, indices, positionMass, gridA);
        CRB_LAUNCHED(2);
        return CRB200_OK;
    }

    // Launch-shape autotuner: each candidate (grid-update CTAs per SM, accumulation and cell-sort
    // CTA counts as multiples of their occupancy) runs `trial` substeps from the same saved state,
    // timed with CUDA events on the solver stream; the fastest stays.  The particle state is
    // restored afterwards and coupling forces of the trials go to scratch, so the caller's
    // simulation is unchanged.
    int Solver::autotune(int trial, int choice[3])
    {
        if (!initialized || stream == nullptr)
        {
            setLastError("autotune: needs an initialized solver on a non-default stream");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        if (trial <= 0)
            trial = 8;
        int dev = 0, sms = 0;
        CRB_CHECK(cudaGetDevice(&dev));
        CRB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const int baseP2g = p2gBase > 0 ? p2gBase : p2gCtas, baseSort = sortBase > 0 ? sortBase : cellCtas;
        p2gBase = baseP2g;
        sortBase = baseSort;
        unsigned char *snap = nullptr;
        CRB_CHECK(cudaMalloc(&snap, stateBytes()));
        if (!adjForce)
        {
            const int ns = std::max(shapes.size, 1);
            CRB_CHECK(cudaMalloc(&adjForce, ns * sizeof(float4)));
            CRB_CHECK(cudaMalloc(&adjTorque, ns * sizeof(float4)));
        }
        int r = saveState(snap);
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (r == CRB200_OK)
            r = cudaFail(cudaEventCreate(&e0), "autotune event");
        if (r == CRB200_OK)
            r = cudaFail(cudaEventCreate(&e1), "autotune event");
        // the resident path (single-scene MLS) tunes the grid update and the fused kernel's CTA
        // multiple; the particle-id path the update, the accumulation and the cell-start kernels
        const bool resident = residentUsable();
        const bool replay0 = adjReplay;
        if (resident)
            scratchCoupling = true;
        else
            adjReplay = true;
        const int upd[3] = {4, 8, 16}, mul[2] = {1, 2};
        float best = 1e30f;
        int bestC[3] = {updCtas / std::max(sms, 1), resident ? resMult : 1, 1};
        for (int a = 0; a < 3 && r == CRB200_OK; ++a)
            for (int b = 0; b < 2 && r == CRB200_OK; ++b)
                for (int c = 0; c < (resident ? 1 : 2) && r == CRB200_OK; ++c)
                {
                    updCtas = sms * upd[a];
                    if (resident)
                        resMult = mul[b];
                    else
                    {
                        p2gCtas = baseP2g * mul[b];
                        cellCtas = baseSort * mul[c];
                    }
                    configVersion++;
                    if ((r = loadState(snap)) != CRB200_OK || (r = stepMany(2)) != CRB200_OK)
                        break; // builds the graph
                    if ((r = loadState(snap)) != CRB200_OK)
                        break;
                    if ((r = cudaFail(cudaEventRecord(e0, stream), "autotune event")) != CRB200_OK)
                        break;
                    if ((r = stepMany(trial)) != CRB200_OK)
                        break;
                    if ((r = cudaFail(cudaEventRecord(e1, stream), "autotune event")) != CRB200_OK)
                        break;
                    float ms = 0.f;
                    if ((r = cudaFail(cudaEventSynchronize(e1), "autotune sync")) != CRB200_OK)
                        break;
                    if ((r = cudaFail(cudaEventElapsedTime(&ms, e0, e1), "autotune timing")) != CRB200_OK)
                        break;
                    if (ms < best)
                    {
                        best = ms;
                        bestC[0] = upd[a];
                        bestC[1] = mul[b];
                        bestC[2] = mul[c];
                    }
                }
        adjReplay = replay0;
        scratchCoupling = false;
        updCtas = sms * bestC[0];
        if (resident)
            resMult = bestC[1];
        else
        {
            p2gCtas = baseP2g * bestC[1];
            cellCtas = baseSort * bestC[2];
        }
        configVersion++;
        if (r == CRB200_OK)
            r = loadState(snap);
        if (r == CRB200_OK)
            r = cudaFail(cudaStreamSynchronize(stream), "autotune sync");
        if (e0)
            cudaEventDestroy(e0);
        if (e1)
            cudaEventDestroy(e1);
        cudaFree(snap);
        if (choice)
        {
            choice[0] = bestC[0];
            choice[1] = bestC[1];
            choice[2] = bestC[2];
        }
        return r;
    }

    // The cell keys and the canonical permutation of the current positions: a sort of them now
    // (the resident path keeps its slots in the order of its last re-sort, which may be older).
    int Solver::copySortState(unsigned *keysOut, unsigned *idsOut)
    {
        const unsigned n = totalParticles();
        if (!n)
            return CRB200_OK;
        if (int r = residentRetire())
            return r;
        if (int r = invalidateRecords())
            return r;
        if (int r = sortParticles(params(), solverType == CRB200_SOLVER_GPU_STANDARD))
            return r;
        if (keysOut)
            CRB_CHECK(cudaMemsetAsync(keysOut, 0xff, n * sizeof(unsigned), stream));
        k_sortKeysOut<<<sortCtas, 64, 0, stream>>>(header, activeList, blockStart, sortedIds, cellStart, keysOut, idsOut);
        CRB_LAUNCHED(1);
        return CRB200_OK;
    }


    int svdBatch(unsigned n, const float *A, float *U, float *V, float *S, float *R, unsigned *fp64Used,
                 unsigned *fp64Count, cudaStream_t stream)
    {
        if (n == 0)
            return CRB200_OK;
        k_svdBatch<<<(n + 127) / 128, 128, 0, stream>>>(n, A, U, V, S, R, fp64Used, fp64Count);
        CRB_LAUNCHED(1);
        return CRB200_OK;
    }

    int Solver::fetchResults()
    {
        if (copiedEvent)
            CRB_CHECK(cudaEventSynchronize(copiedEvent));
        CRB_CHECK(cudaStreamSynchronize(stream));
        return CRB200_OK;
    }
} // namespace crb200

#include "resident_host.cuh"
#include "adjoint.cuh"
