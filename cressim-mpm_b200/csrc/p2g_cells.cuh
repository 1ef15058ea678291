// P2G with one thread per grid cell (included by mpm_kernels.cu).
//
// One 64-thread CTA takes one 4x4x4-cell block of the sorted particle list:
//   1. the block's cell ranges come from the per-cell starts of the sort;
//   2. thread c walks the particles of cell c in sorted order, loading each one a particle ahead,
//      turns it into the affine contribution u + i*a0 + j*a1 + k*a2 (MLS / PB-MPM) and
//      accumulates the 27 stencil nodes in registers (the sums inside a block are deterministic);
//   3. a 27-phase flush adds the registers into a per-warp shared-memory 6x6x6 node tile: in one
//      phase the 32 lanes of a warp write 32 distinct nodes, so no atomics are needed;
//   4. the two warp tiles are summed in a fixed order and each touched node gets one float4
//      vector atomic in the block-major accumulation grid.
// Particles whose stencil base lies outside the grid take a per-particle path with global vector
// atomics instead, and particles beyond the first kCellRun of a cell are added by vector atomics.
#pragma once

namespace crb200
{
    constexpr int kRec = 16;       // floats per staged particle
    constexpr int kCellRun = 9;    // particles a cell thread accumulates; the rest of a cell's
                                   // particles go through per-particle vector atomics

    // Per-particle scatter with global vector atomics (outliers and oversized blocks).
    // Mode 0 MLS, 1 PB (u/a already include the mass), 2 standard momentum, 3 standard force.
    template <int Mode>
    __device__ __forceinline__ void scatterGlobal(const StepParams &p, const Stencil &st, const float *rec,
                                                  unsigned cutMask, float4 *__restrict__ gridA, float4 *__restrict__ gridF)
    {
        const GridGeom &g = p.g;
        float w[3][3], dw[3][3];
        weights(st.fx, w);
        if (Mode == 3)
            weightGrads(st.fx, dw);
        const V3 u = v3(rec[0], rec[1], rec[2]);
        const float m = rec[3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int k = 0; k < 3; ++k)
                {
                    const int ni = st.b[0] + i, nj = st.b[1] + j, nk = st.b[2] + k;
                    if (!inGrid(g, ni, nj, nk) || ((cutMask >> (i * 9 + j * 3 + k)) & 1u))
                        continue;
                    const float wt = w[i][0] * w[j][1] * w[k][2];
                    const unsigned a = nodeAddr(g, ni, nj, nk);
                    if (Mode == 3)
                    {
                        const V3 gw = v3(dw[i][0] * w[j][1] * w[k][2], w[i][0] * dw[j][1] * w[k][2],
                                         w[i][0] * w[j][1] * dw[k][2]);
                        const float wm = wt * m;
                        const V3 f = v3(p.gravity.x * wm + rec[4] * gw.x + rec[7] * gw.y + rec[10] * gw.z,
                                        p.gravity.y * wm + rec[5] * gw.x + rec[8] * gw.y + rec[11] * gw.z,
                                        p.gravity.z * wm + rec[6] * gw.x + rec[9] * gw.y + rec[12] * gw.z);
                        atomicAdd(&gridF[a], make_float4(f.x, f.y, f.z, 0.f));
                    }
                    else
                    {
                        V3 val = u;
                        if (Mode <= 1)
                            val = u + v3(rec[4], rec[5], rec[6]) * (float)i + v3(rec[7], rec[8], rec[9]) * (float)j +
                                  v3(rec[10], rec[11], rec[12]) * (float)k;
                        atomicAdd(&gridA[a], make_float4(val.x * wt, val.y * wt, val.z * wt, m * wt));
                    }
                }
    }

    // Raw particle data a P2G thread needs (loaded one particle ahead of its use).
    struct RawParticle
    {
        float4 x4, v4, mp;
        float F[9], C[9];
        float v0;
        int mt;
    };

    template <int Mode>
    __device__ __forceinline__ void loadRaw(unsigned id, const float4 *__restrict__ xm, const float4 *__restrict__ vel,
                                            const float4 *__restrict__ matParams, const int *__restrict__ matType,
                                            const float *__restrict__ F, const float *__restrict__ Cm,
                                            const float *__restrict__ V0, unsigned stride, RawParticle &r)
    {
        r.x4 = xm[id];
        r.v4 = vel[id];
        r.mp = matParams[id];
        r.mt = matType[id];
#pragma unroll
        for (int k = 0; k < 9; ++k)
            r.F[k] = F[k * stride + id];
        if (Mode != 2)
        {
#pragma unroll
            for (int k = 0; k < 9; ++k)
                r.C[k] = Cm[k * stride + id];
        }
        r.v0 = (Mode == 1) ? 0.f : V0[id];
    }

    // Record of one particle for the cell accumulation:
    //   [0..2] u, [3] m, [4..12] a0 a1 a2 (MLS / PB) or -V0*tau column-major (standard force),
    //   [13..15] fx.
    // Returns false when the particle must not go through the cell path (non-finite position or a
    // stencil base outside [0, n-2]); such particles are scattered here with global atomics when
    // scatterOutliers is set.
    template <int Mode>
    __device__ __forceinline__ bool buildRecord(const StepParams &p, unsigned id, const RawParticle &raw,
                                                float *__restrict__ Cm, unsigned stride, unsigned cutMask,
                                                bool scatterOutliers, float4 *__restrict__ gridA,
                                                float4 *__restrict__ gridF, unsigned *fp64Count, float rec[kRec])
    {
        const GridGeom &g = p.g;
        const Stencil st = stencilOf(g, v3(raw.x4));
        const float m = raw.x4.w;
#pragma unroll
        for (int e = 0; e < kRec; ++e)
            rec[e] = 0.f;
        if (!st.finite)
            return false;
        const V3 v = v3(raw.v4);
        M3 Fp;
#pragma unroll
        for (int e = 0; e < 9; ++e)
            Fp.m[e] = raw.F[e];
        const float dx = g.dx;
        if (Mode == 0 || Mode == 1)
        {
            M3 A, Cp;
#pragma unroll
            for (int e = 0; e < 9; ++e)
                Cp.m[e] = raw.C[e];
            V3 base;
            if (Mode == 0)
            {
                const M3 s = kirchhoffStress(Fp, raw.mp.x, raw.mp.y, raw.mt);
                const float coef = -p.dt * 4.f * g.invDx * g.invDx * raw.v0;
#pragma unroll
                for (int e = 0; e < 9; ++e)
                    A.m[e] = s.m[e] * coef + Cp.m[e] * m;
                base = (v + v3(p.gravity) * p.dt) * m;
            }
            else
            {
                if (raw.mt == 1 || raw.mt == 0)
                {
                    // solveMaterialConstraints (constitutive_models.h:123-156)
                    M3 tF;
#pragma unroll
                    for (int e = 0; e < 9; ++e)
                        tF.m[e] = Cp.m[e] * p.dt + ((e % 4) == 0 ? 1.f : 0.f);
                    tF = matmul(tF, Fp);
                    const M3 R = pbRotationTarget(tF, fp64Count);
                    const float detF = det3(tF);
                    const float cd = fminf(fmaxf(fabsf(detF), 0.1f), 1000.0f);
                    const float qs = 1.0f / (copysignf(1.0f, detF) * sqrtf(cd));
                    M3 tgt;
#pragma unroll
                    for (int e = 0; e < 9; ++e)
                        tgt.m[e] = R.m[e] * raw.mp.y + (tF.m[e] * qs) * (1.0f - raw.mp.y);
                    const M3 TF = matmul(tgt, inverse3(Fp));
#pragma unroll
                    for (int e = 0; e < 9; ++e)
                        Cp.m[e] = Cp.m[e] + ((TF.m[e] - ((e % 4) == 0 ? 1.f : 0.f)) - Cp.m[e] * p.dt) * raw.mp.x;
                    storeM3(Cm, stride, id, Cp);
                }
#pragma unroll
                for (int e = 0; e < 9; ++e)
                    A.m[e] = Cp.m[e] * m;
                base = v * m;
            }
            // u = base - A (fx dx); a_c = dx * A column c
            const V3 fd = v3(st.fx.x * dx, st.fx.y * dx, st.fx.z * dx);
            rec[0] = base.x - (A.m[0] * fd.x + A.m[3] * fd.y + A.m[6] * fd.z);
            rec[1] = base.y - (A.m[1] * fd.x + A.m[4] * fd.y + A.m[7] * fd.z);
            rec[2] = base.z - (A.m[2] * fd.x + A.m[5] * fd.y + A.m[8] * fd.z);
#pragma unroll
            for (int e = 0; e < 9; ++e)
                rec[4 + e] = A.m[e] * dx;
        }
        else
        {
            // standard MPM: momentum v m, force -V0 tau grad w + g w m (standard_mpm_algorithm.h:166-206)
            const M3 s = kirchhoffStress(Fp, raw.mp.x, raw.mp.y, raw.mt);
            const float nv0 = -raw.v0;
            rec[0] = v.x * m;
            rec[1] = v.y * m;
            rec[2] = v.z * m;
#pragma unroll
            for (int e = 0; e < 9; ++e)
                rec[4 + e] = s.m[e] * nv0;
        }
        rec[3] = m;
        rec[13] = st.fx.x;
        rec[14] = st.fx.y;
        rec[15] = st.fx.z;
        const bool inside = st.b[0] >= 0 && st.b[0] <= g.n.x - 2 && st.b[1] >= 0 && st.b[1] <= g.n.y - 2 &&
                            st.b[2] >= 0 && st.b[2] <= g.n.z - 2;
        if (!inside)
        {
            if (!scatterOutliers)
                return false;
            if (Mode == 2)
            {
                scatterGlobal<2>(p, st, rec, 0u, gridA, gridF);
                scatterGlobal<3>(p, st, rec, 0u, gridA, gridF);
            }
            else
                scatterGlobal<Mode>(p, st, rec, cutMask, gridA, gridF);
            return false;
        }
        return true;
    }

    // Adds one particle's 27 node contributions to the cell thread's registers.
    template <int Mode, bool Masked>
    __device__ __forceinline__ void accumulateCell(const StepParams &p, const float rec[kRec], unsigned msk, int pass,
                                                   float acc[27][4])
    {
        const V3 u = v3(rec[0], rec[1], rec[2]);
        const float m = rec[3];
        const V3 a0 = v3(rec[4], rec[5], rec[6]);
        const V3 a1 = v3(rec[7], rec[8], rec[9]);
        const V3 a2 = v3(rec[10], rec[11], rec[12]);
        const V3 fx = v3(rec[13], rec[14], rec[15]);
        float w[3][3], dw[3][3];
        weights(fx, w);
        if (Mode == 2 && pass == 1)
            weightGrads(fx, dw);
#pragma unroll
        for (int i = 0; i < 3; ++i)
        {
            const V3 ui = i == 0 ? u : fma3(a0, (float)i, u);
#pragma unroll
            for (int j = 0; j < 3; ++j)
            {
                const V3 uij = j == 0 ? ui : fma3(a1, (float)j, ui);
                const float wij = w[i][0] * w[j][1];
#pragma unroll
                for (int k = 0; k < 3; ++k)
                {
                    const int n = i * 9 + j * 3 + k;
                    if (Masked && ((msk >> n) & 1u))
                        continue;
                    const float wt = wij * w[k][2];
                    if (Mode == 2 && pass == 1)
                    {
                        const float wm = wt * m;
                        const float gx = dw[i][0] * w[j][1] * w[k][2], gy = w[i][0] * dw[j][1] * w[k][2],
                                    gz = wij * dw[k][2];
                        acc[n][0] += p.gravity.x * wm + a0.x * gx + a1.x * gy + a2.x * gz;
                        acc[n][1] += p.gravity.y * wm + a0.y * gx + a1.y * gy + a2.y * gz;
                        acc[n][2] += p.gravity.z * wm + a0.z * gx + a1.z * gy + a2.z * gz;
                    }
                    else if (Mode == 2)
                    {
                        acc[n][0] += u.x * wt;
                        acc[n][1] += u.y * wt;
                        acc[n][2] += u.z * wt;
                        acc[n][3] += m * wt;
                    }
                    else
                        fma4acc(acc[n], k == 0 ? uij : fma3(a2, (float)k, uij), m, wt);
                }
            }
        }
    }

    // (b) One record per particle (indexed by particle id), particle-parallel over the sorted slots.
    //     Outliers are scattered here with global atomics and leave a zero record.  PB-MPM's
    //     material constraint writes the relaxed C back.  Nothing to do when the previous substep's
    //     G2P already wrote the records (hdr->recordsValid; PB-MPM: hdr->pbRecordsValid).
    template <int Mode, bool Multi>
    __global__ void __launch_bounds__(128, Mode == 1 ? 4 : 8) k_record(const __grid_constant__ StepParams p0, SceneTable sc,
                                                    const SortHeader *__restrict__ hdr,
                                                    const unsigned *__restrict__ sortedIds, const float4 *__restrict__ xm,
                                                    const float4 *__restrict__ vel, const float4 *__restrict__ matParams,
                                                    const int *__restrict__ matType, const float *__restrict__ F,
                                                    float *__restrict__ Cm, const float *__restrict__ V0, unsigned stride,
                                                    const unsigned *__restrict__ cutMasks, float4 *__restrict__ records,
                                                    float4 *__restrict__ gridA, float4 *__restrict__ gridF, unsigned *fp64Count)
    {
        if ((Mode == 0 && !Multi && hdr->recordsValid) || (Mode == 1 && hdr->pbRecordsValid))
            return;
        const bool carry = Mode == 0 && Multi && hdr->recordsValid;
        const unsigned nS = hdr->numSorted;
        for (unsigned j = blockIdx.x * blockDim.x + threadIdx.x; j < nS; j += gridDim.x * blockDim.x)
        {
        const unsigned id = sortedIds[j];
        const unsigned si = Multi ? sc.particleScene[id] : 0u; // sorted particles have a scene
        if (carry && !(sc.flags[si] & SF_SLICER))
            continue; // the previous G2P wrote this particle's record
        const StepParams &p = Multi ? sc.params[si] : p0;
        const bool slicers = Mode <= 1 && p.numShapes > 0 && (sc.flags[si] & SF_SLICER);
        const unsigned msk = slicers ? cutMasks[id] : 0u;
        RawParticle raw;
        loadRaw<Mode>(id, xm, vel, matParams, matType, F, Cm, V0, stride, raw);
        float rec[kRec];
        if (!buildRecord<Mode>(p, id, raw, Cm, stride, msk, true, gridA, gridF, fp64Count, rec))
        {
#pragma unroll
            for (int e = 0; e < kRec; ++e)
                rec[e] = 0.f;
        }
        float4 *out = records + 4ull * id;
        out[0] = make_float4(rec[0], rec[1], rec[2], rec[3]);
        out[1] = make_float4(rec[4], rec[5], rec[6], rec[7]);
        out[2] = make_float4(rec[8], rec[9], rec[10], rec[11]);
        out[3] = make_float4(rec[12], rec[13], rec[14], rec[15]);
        }
    }

    __device__ __forceinline__ void loadRecord(const float4 *__restrict__ records, unsigned j, float rec[kRec])
    {
        const float4 *r = records + 4ull * j;
        const float4 a = __ldg(r), b = __ldg(r + 1), c = __ldg(r + 2), d = __ldg(r + 3);
        rec[0] = a.x; rec[1] = a.y; rec[2] = a.z; rec[3] = a.w;
        rec[4] = b.x; rec[5] = b.y; rec[6] = b.z; rec[7] = b.w;
        rec[8] = c.x; rec[9] = c.y; rec[10] = c.z; rec[11] = c.w;
        rec[12] = d.x; rec[13] = d.y; rec[14] = d.z; rec[15] = d.w;
    }

    // (c) Cell accumulation: one 64-thread CTA per active block, one thread per cell.
    //     Multi: each active block reads its scene's parameters (block base search).
    //     Det: nothing is added atomically.  A cell thread accumulates all of its cell's particles
    //     (no kCellRun cap) and the block's whole 6x6x6 tile is stored to tiles[block] (tilesF for
    //     the standard solver's force pass), from which the grid update sums each node's sources in
    //     a fixed order.
    template <int Mode, bool Multi, bool Det = false>
    __global__ void __launch_bounds__(64, Multi ? 5 : 6) k_accumulate(const __grid_constant__ StepParams p0, SceneTable sc, const SortHeader *__restrict__ hdr,
                                                       const unsigned *__restrict__ activeList,
                                                       const unsigned *__restrict__ blockStart,
                                                       const unsigned *__restrict__ sortedIds,
                                                       const unsigned *__restrict__ cellStart,
                                                       const float4 *__restrict__ records,
                                                       const unsigned *__restrict__ cutMasks, float4 *__restrict__ gridA,
                                                       float4 *__restrict__ gridF, float4 *__restrict__ tiles = nullptr,
                                                       float4 *__restrict__ tilesF = nullptr)
    {
        __shared__ unsigned sStart[65];
        __shared__ unsigned sOv[65];
        __shared__ unsigned sWarpTot;
        __shared__ float sTile[2][4 * kTileNodes];
        __shared__ StepParams sP; // Multi: the current block's scene parameters

        const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
        const int passes = Mode == 2 ? 2 : 1;
        for (int t = tid; t < 2 * 4 * kTileNodes; t += 64)
            (&sTile[0][0])[t] = 0.f;
        const unsigned nAct = hdr->numActiveBlocks;
        const int cx = tid & 3, cy = (tid >> 2) & 3, cz = tid >> 4;
        for (unsigned ab = blockIdx.x; ab < nAct; ab += gridDim.x)
        {
            const unsigned b = activeList[ab];
            const unsigned si = Multi ? (unsigned)sceneOfBlock(sc, b) : 0u;
            if (Multi)
            {
                // read at the use sites from shared memory rather than held in registers
                constexpr int words = (int)(sizeof(StepParams) / sizeof(unsigned));
                static_assert(words <= 64, "StepParams must fit one load per thread");
                if (tid < words)
                    reinterpret_cast<unsigned *>(&sP)[tid] = reinterpret_cast<const unsigned *>(&sc.params[si])[tid];
                __syncthreads();
            }
            const StepParams &p = Multi ? sP : p0;
            const GridGeom &g = p.g;
            const bool slicers = Mode <= 1 && p.numShapes > 0 && (sc.flags[si] & SF_SLICER);
            const unsigned lb = b - g.blockBase;
            const int bx = lb % g.nb.x, by = (lb / g.nb.x) % g.nb.y, bz = lb / (g.nb.x * g.nb.y);
            const unsigned start = blockStart[b], cnt = blockStart[b + 1] - start;
            // cell ranges of this block's sorted slots (cells are contiguous, in cell order)
            {
                const unsigned excl = cellStart[b * 64u + tid] - start;
                const unsigned v = (tid < 63 ? cellStart[b * 64u + tid + 1] - start : cnt) - excl;
                sStart[tid] = excl;
                if (tid == 63)
                    sStart[64] = cnt;
                // overflow prefix: particles beyond the first kCellRun of each cell
                const unsigned ov = v > (unsigned)kCellRun ? v - (unsigned)kCellRun : 0u;
                unsigned oinc = ov;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1)
                {
                    const unsigned y = __shfl_up_sync(0xffffffffu, oinc, o);
                    if (lane >= o)
                        oinc += y;
                }
                __syncthreads();
                if (tid == 31)
                    sWarpTot = oinc;
                __syncthreads();
                sOv[tid + 1] = oinc + (warp ? sWarpTot : 0u);
                if (tid == 0)
                    sOv[0] = 0;
            }
            __syncthreads();
            const unsigned cs = sStart[tid], ce = sStart[tid + 1];
            // Det: a cell thread takes all of its cell's particles, so nothing goes through atomics
            const unsigned runEnd = Det ? ce : min(ce, cs + (unsigned)kCellRun);
            for (int pass = 0; pass < passes; ++pass)
            {
                float acc[27][4];
#pragma unroll
                for (int n = 0; n < 27; ++n)
                {
                    acc[n][0] = 0.f;
                    acc[n][1] = 0.f;
                    acc[n][2] = 0.f;
                    acc[n][3] = 0.f;
                }
                float nxt[kRec];
                unsigned nid = cs < runEnd ? sortedIds[start + cs] : 0u;
                if (cs < runEnd)
                    loadRecord(records, nid, nxt);
                for (unsigned q = cs; q < runEnd; ++q)
                {
                    float rec[kRec];
#pragma unroll
                    for (int e = 0; e < kRec; ++e)
                        rec[e] = nxt[e];
                    const unsigned id = nid;
                    if (q + 1 < runEnd)
                    {
                        nid = sortedIds[start + q + 1];
                        loadRecord(records, nid, nxt);
                    }
                    if (q + 2 < runEnd)
                    {
                        // the record after next into L1 (no registers held for it)
                        const float4 *ahead = records + 4ull * sortedIds[start + q + 2];
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(ahead));
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(ahead + 2));
                    }
                    const unsigned msk = slicers ? cutMasks[id] : 0u;
                    if (msk)
                        accumulateCell<Mode, true>(p, rec, msk, pass, acc);
                    else
                        accumulateCell<Mode, false>(p, rec, 0u, pass, acc);
                }
                // phased flush of the registers into this warp's tile
                float *tile = sTile[warp];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j)
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                        {
                            const int n = i * 9 + j * 3 + k;
                            const int t = (cx + i) + kTileEdge * ((cy + j) + kTileEdge * (cz + k));
                            tile[t] += acc[n][3];
                            tile[kTileNodes + t] += acc[n][0];
                            tile[2 * kTileNodes + t] += acc[n][1];
                            tile[3 * kTileNodes + t] += acc[n][2];
                            __syncwarp();
                        }
                __syncthreads();
                // fixed-order sum of the warp tiles, one vector atomic per touched node
                for (int t = tid; t < kTileNodes; t += 64)
                {
                    const float m = sTile[0][t] + sTile[1][t];
                    const float px = sTile[0][kTileNodes + t] + sTile[1][kTileNodes + t];
                    const float py = sTile[0][2 * kTileNodes + t] + sTile[1][2 * kTileNodes + t];
                    const float pz = sTile[0][3 * kTileNodes + t] + sTile[1][3 * kTileNodes + t];
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                    {
                        sTile[0][c * kTileNodes + t] = 0.f;
                        sTile[1][c * kTileNodes + t] = 0.f;
                    }
                    if (Det)
                    {
                        float4 *dst = (Mode == 2 && pass == 1) ? tilesF : tiles;
                        dst[(size_t)b * kTileNodes + t] = make_float4(px, py, pz, m);
                        continue;
                    }
                    const int tx = t % kTileEdge, ty = (t / kTileEdge) % kTileEdge, tz = t / (kTileEdge * kTileEdge);
                    const int i = 4 * bx + tx, j = 4 * by + ty, k = 4 * bz + tz;
                    if (!inGrid(g, i, j, k))
                        continue;
                    const unsigned a = nodeAddr(g, i, j, k);
                    if (Mode == 2 && pass == 1)
                    {
                        if (px != 0.f || py != 0.f || pz != 0.f)
                            atomicAdd(&gridF[a], make_float4(px, py, pz, 0.f));
                    }
                    else if (m != 0.f || px != 0.f || py != 0.f || pz != 0.f)
                        atomicAdd(&gridA[a], make_float4(px, py, pz, m));
                }
                // particles beyond the first kCellRun of a cell: one per thread, vector atomics
                const unsigned total = Det ? 0u : sOv[64];
                for (unsigned kk = tid; kk < total; kk += 64)
                {
                    int lo = 0, hi = 63;
                    while (lo < hi)
                    {
                        const int mid = (lo + hi + 1) >> 1;
                        if (sOv[mid] <= kk)
                            lo = mid;
                        else
                            hi = mid - 1;
                    }
                    const unsigned slot = start + sStart[lo] + (unsigned)kCellRun + (kk - sOv[lo]);
                    float rec[kRec];
                    const unsigned sid = sortedIds[slot];
                    loadRecord(records, sid, rec);
                    if (rec[3] == 0.f && rec[0] == 0.f && rec[1] == 0.f && rec[2] == 0.f)
                        continue; // zero record (outlier already scattered, or massless)
                    Stencil st;
                    st.b[0] = 4 * bx + (lo & 3);
                    st.b[1] = 4 * by + ((lo >> 2) & 3);
                    st.b[2] = 4 * bz + (lo >> 4);
                    st.fx = v3(rec[13], rec[14], rec[15]);
                    st.finite = true;
                    const unsigned msk = slicers ? cutMasks[sid] : 0u;
                    if (Mode == 2 && pass == 0)
                        scatterGlobal<2>(p, st, rec, 0u, gridA, gridF);
                    else if (Mode == 2)
                        scatterGlobal<3>(p, st, rec, 0u, gridA, gridF);
                    else
                        scatterGlobal<Mode>(p, st, rec, msk, gridA, gridF);
                }
                __syncthreads();
            }
        }
    }
} // namespace crb200
