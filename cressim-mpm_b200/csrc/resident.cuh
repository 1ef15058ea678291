// Resident cell-ordered particle state and the fused G2P -> P2G substep (single-scene MLS-MPM;
// included by mpm_kernels.cu).
//
// The particle-id-ordered path reads every particle twice per substep (G2P, then the P2G of the
// next substep through a 64-byte record) and sorts the particles every substep.  Here the solver
// keeps its own copy of the particle state in slots grouped by 4x4x4 grid block and cell, and one
// kernel per substep does, block by block:
//   1. stage the block's 8x8x8 node window of grid velocities in shared memory (nodes 4b-1 ..
//      4b+6 per axis: every stencil of a particle whose base cell is within one cell of the block);
//   2. per particle (slot order, coalesced): G2P from the window (the reference's
//      mls_mpm_algorithm.h:296-390), the particle update, then the next substep's P2G record
//      (mls_mpm_algorithm.h:147-241) of the updated particle;
//   3. records of particles whose (new) cell lies in the block go to shared memory by (rank in
//      cell, cell), the rank from a shared counter per cell; 192 threads, one per (cell, x-slab of
//      the 3x3x3 stencil), add their cell's records into registers and reduce those sums into a
//      shared 8x8x8 output window;
//   4. particles that moved out of the block, left the window (or the grid) or come beyond a
//      cell's kResRanks are added with global vector atomics (fire-and-forget reductions);
//   5. the output window goes to the accumulation grid with one float4 vector atomic per node that
//      received mass, and the grid blocks it touched are appended to the touched-block list the
//      grid update walks.
// Per substep each particle's position and F are read and written once and its V0 read; C is
// written only by the last substep of a call, which also writes the velocities to the caller's
// buffer.  The slots are re-sorted at the start of a call only when the previous call left
// particles outside their block's window or too many outside their block; correctness never
// depends on the grouping, only the share of particles that take the slower paths does.
#pragma once

namespace crb200
{
    constexpr int kResThreads = 192;    // 64 cells x 3 x-slabs in the accumulation phase
    constexpr int kResRanks = 12;       // particles per cell accumulated from shared records
    constexpr int kResRecStride = 65;   // record (rank k, cell c) at k * 65 + c: conflict-free banks
    constexpr int kResRecCh = kResRanks * kResRecStride;
    constexpr int kWinNodes = 512;      // 8 x 8 x 8 node window, origin 4b - 1 per axis
    constexpr int kOutZ = 68;           // z stride of the output window (spreads a warp's cells over the banks)
    constexpr int kOutCh = 8 * kOutZ;   // floats per output channel

    struct ResShared
    {
        float4 gv[kWinNodes];        // grid velocities of the window (x + 8 y + 64 z)
        float out[4][kOutCh];        // momentum xyz, mass of the next grid (x + 8 y + 68 z)
        float rec[kRec][kResRecCh];  // records of the block's particles by (rank, cell)
        unsigned count[64];          // particles of each cell of the block (rank counters)
        unsigned range[2];           // the block's slots
        unsigned touchedBits, movers, outside, pad0, pad1, pad2;
    };
    static_assert(sizeof(ResShared) % 16 == 0, "shapes follow ResShared in shared memory");

    __device__ __forceinline__ void markTouched(unsigned blk, unsigned *__restrict__ touchedFlag,
                                                unsigned *__restrict__ touchedList, SortHeader *hdr)
    {
        if (atomicExch(&touchedFlag[blk], 1u) == 0u)
            touchedList[atomicAdd(&hdr->numTouchedBlocks, 1u)] = blk;
    }

    // A record passed by value, so that the caller's copy stays in registers.
    struct RecVal
    {
        float r[kRec];
    };

    // One particle's record scattered with global vector atomics (bounds-checked, slicer-masked),
    // each touched grid block listed for the grid update.  Out of line: rare.
    __device__ __noinline__ void resScatterGlobal(GridGeom g, Stencil st, RecVal rv, unsigned msk,
                                                  float4 *__restrict__ gridA, unsigned *__restrict__ touchedFlag,
                                                  unsigned *__restrict__ touchedList, SortHeader *hdr)
    {
        const float *rec = rv.r;
        float w[3][3];
        weights(st.fx, w);
        const V3 u = v3(rec[0], rec[1], rec[2]);
        const V3 a0 = v3(rec[4], rec[5], rec[6]), a1 = v3(rec[7], rec[8], rec[9]), a2 = v3(rec[10], rec[11], rec[12]);
        const float m = rec[3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k)
                {
                    const int ni = st.b[0] + i, nj = st.b[1] + j, nk = st.b[2] + k;
                    if (!inGrid(g, ni, nj, nk) || ((msk >> (i * 9 + j * 3 + k)) & 1u))
                        continue;
                    const float wt = (w[i][0] * w[j][1]) * w[k][2];
                    const V3 val = ((u + a0 * (float)i) + a1 * (float)j) + a2 * (float)k;
                    atomicAdd(&gridA[nodeAddr(g, ni, nj, nk)], make_float4(val.x * wt, val.y * wt, val.z * wt, m * wt));
                    markTouched(g.blockBase + (unsigned)((ni >> 2) + g.nb.x * ((nj >> 2) + g.nb.y * (nk >> 2))),
                                touchedFlag, touchedList, hdr);
                }
    }

    // One particle's record added straight to the accumulation grid with one float4 vector
    // reduction per in-grid node not cut off by a slicer (a crowded cell's particles beyond
    // kResRanks, and particles that left their block but not its window).  Fire-and-forget
    // reductions keep the warp moving; the caller has the blocks listed for the grid update.
    __device__ __forceinline__ void resScatterRed(const GridGeom &g, const Stencil &st, const float *rec, unsigned msk,
                                                  float4 *__restrict__ gridA)
    {
        float w[3][3];
        weights(st.fx, w);
        const V3 u = v3(rec[0], rec[1], rec[2]);
        const V3 a0 = v3(rec[4], rec[5], rec[6]), a1 = v3(rec[7], rec[8], rec[9]), a2 = v3(rec[10], rec[11], rec[12]);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int k = 0; k < 3; ++k)
                {
                    const int ni = st.b[0] + i, nj = st.b[1] + j, nk = st.b[2] + k;
                    if (!inGrid(g, ni, nj, nk) || ((msk >> (i * 9 + j * 3 + k)) & 1u))
                        continue;
                    const float wt = (w[i][0] * w[j][1]) * w[k][2];
                    const V3 val = ((u + a0 * (float)i) + a1 * (float)j) + a2 * (float)k;
                    atomicAdd(&gridA[nodeAddr(g, ni, nj, nk)], make_float4(val.x * wt, val.y * wt, val.z * wt, rec[3] * wt));
                }
    }

    // The fused substep kernel.  DoG2P: G2P of the current substep from the grid velocities.
    // DoP2G: P2G of the next substep into the accumulation grid.  Export (with DoG2P, without DoP2G,
    // the last substep of a call): positions and velocities go to the caller's particle-id-ordered
    // buffers instead of the resident ones.  Without DoG2P (the first substep of a call) positions
    // and velocities come from the caller's buffers, so edits made between calls are honoured.
    template <bool DoG2P, bool DoP2G, bool Export>
    __global__ void __launch_bounds__(kResThreads, 3)
        k_g2p2g(const __grid_constant__ StepParams p, SortHeader *hdr, const unsigned *__restrict__ activeList,
                const unsigned *__restrict__ blockStart, ResState rs, float4 *callerX, float4 *callerV,
                const float4 *__restrict__ gridV, float4 *__restrict__ gridA, unsigned *__restrict__ touchedFlag,
                unsigned *__restrict__ touchedList, const ShapeRec *__restrict__ shapeTable, SdfPtrs sdf,
                const unsigned long long *__restrict__ blockShapeMask, const unsigned *__restrict__ sceneFlags)
    {
        extern __shared__ float4 resSmem4[];
        ResShared &S = *reinterpret_cast<ResShared *>(resSmem4);
        ShapeRec *shp = reinterpret_cast<ShapeRec *>(reinterpret_cast<unsigned char *>(resSmem4) + sizeof(ResShared));
        const int tid = threadIdx.x;
        const GridGeom &g = p.g;
        if (p.numShapes > 0)
            loadShapes(shp, shapeTable, p.numShapes);
        if (tid == 0)
        {
            S.movers = 0u;
            S.outside = 0u;
        }
        if (DoP2G)
        {
            for (int t = tid; t < 4 * kOutCh; t += kResThreads)
                (&S.out[0][0])[t] = 0.f;
            if (tid < 64)
                S.count[tid] = 0u;
        }
        const bool slicers = p.numShapes > 0 && (sceneFlags[0] & SF_SLICER);
        const bool mixed = hdr->matMixed != 0u;
        const float4 matU = hdr->matUniform;
        const unsigned nAct = hdr->numActiveBlocks;
        for (unsigned ab = blockIdx.x; ab < nAct; ab += gridDim.x)
        {
            const unsigned b = activeList[ab];
            const unsigned lb = b - g.blockBase;
            const int bx = (int)(lb % (unsigned)g.nb.x), by = (int)((lb / (unsigned)g.nb.x) % (unsigned)g.nb.y),
                      bz = (int)(lb / (unsigned)(g.nb.x * g.nb.y));
            const int ox = 4 * bx - 1, oy = 4 * by - 1, oz = 4 * bz - 1;
            __syncthreads(); // the previous block is done with the windows and the counters
            if (tid == 0)
                S.range[0] = blockStart[b];
            else if (tid == 1)
                S.range[1] = blockStart[b + 1];
            else if (tid == 2)
                S.touchedBits = 0u;
            if (DoG2P)
                for (int t = tid; t < kWinNodes; t += kResThreads)
                {
                    const int i = ox + (t & 7), j = oy + ((t >> 3) & 7), k = oz + (t >> 6);
                    S.gv[t] = inGrid(g, i, j, k) ? gridV[nodeAddr(g, i, j, k)] : make_float4(0.f, 0.f, 0.f, 0.f);
                }
            __syncthreads();
            const unsigned s0 = S.range[0], s1 = S.range[1];
            // ---- particles, in slot order
            for (unsigned s = s0 + (unsigned)tid; s < s1; s += kResThreads)
            {
                // the particle id only where the caller's buffers are read or written
                const unsigned id = (!DoG2P || Export) ? rs.id[s] : 0u;
                float4 x4;
                V3 v = v3(0.f, 0.f, 0.f);
                if (DoG2P)
                {
                    x4 = rs.x[s];
                    if (slicers) // G2P of a cut particle falls back on its own velocity
                        v = v3(rs.v[s]);
                }
                else
                {
                    x4 = callerX[id];
                    v = v3(callerV[id]);
                    rs.x[s] = x4;
                    if (slicers)
                        rs.v[s] = make_float4(v.x, v.y, v.z, 0.f);
                }
                const float V0p = rs.V0[s];
                M3 Fp, Cp;
                loadM3(rs.F, rs.stride, s, Fp);
                if (!DoG2P)
                    loadM3(rs.C, rs.stride, s, Cp);
                V3 x = v3(x4);
                if (DoG2P)
                {
                    const Stencil st = stencilOf(g, x);
                    float w[3][3];
                    weights(st.fx, w);
                    const unsigned msk = slicers ? rs.cut[s] : 0u;
                    V3 Sv = v3(0.f, 0.f, 0.f);
                    float T[9];
#pragma unroll
                    for (int e = 0; e < 9; ++e)
                        T[e] = 0.f;
                    if (st.finite)
                    {
                        const int rx = st.b[0] - ox, ry = st.b[1] - oy, rz = st.b[2] - oz;
                        const bool interior = st.b[0] >= 0 && st.b[0] <= g.n.x - 3 && st.b[1] >= 0 &&
                                              st.b[1] <= g.n.y - 3 && st.b[2] >= 0 && st.b[2] <= g.n.z - 3;
                        if (interior && msk == 0u && rx >= 0 && rx <= 5 && ry >= 0 && ry <= 5 && rz >= 0 && rz <= 5)
                        {
                            // the separable contraction of k_g2p, from the window
#pragma unroll
                            for (int a = 0; a < 3; ++a)
                            {
                                V3 Y = v3(0.f, 0.f, 0.f), Yb = v3(0.f, 0.f, 0.f), Yc = v3(0.f, 0.f, 0.f);
#pragma unroll
                                for (int bb = 0; bb < 3; ++bb)
                                {
                                    const int t = (rx + a) + 8 * (ry + bb) + 64 * rz;
                                    const V3 v0 = v3(S.gv[t]), v1 = v3(S.gv[t + 64]), v2 = v3(S.gv[t + 128]);
                                    const V3 Zc = fma3(v2, 2.f * w[2][2], mul3(v1, w[1][2]));
                                    const V3 Z = fma3(v2, w[2][2], fma3(v1, w[1][2], mul3(v0, w[0][2])));
                                    Y = fma3(Z, w[bb][1], Y);
                                    if (bb)
                                        Yb = fma3(Z, (float)bb * w[bb][1], Yb);
                                    Yc = fma3(Zc, w[bb][1], Yc);
                                }
                                const V3 wY = Y * w[a][0];
                                Sv = Sv + wY;
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
                        else
                        {
                            G2PWeights W;
#pragma unroll
                            for (int q = 0; q < 3; ++q)
#pragma unroll
                                for (int d = 0; d < 3; ++d)
                                {
                                    W.w[q][d] = w[q][d];
                                    W.dw[q][d] = 0.f;
                                }
                            const V3 vk = msk ? v + v3(p.gravity) * p.dt : v3(0.f, 0.f, 0.f);
                            const G2PMoments r = g2pGatherGeneral<0>(g, st, x, vk, msk, W, shp, p.numShapes, sdf, gridV);
                            Sv = r.S;
#pragma unroll
                            for (int e = 0; e < 9; ++e)
                                T[e] = r.T[e];
                        }
                    }
                    M3 Cn;
                    {
                        const float s4 = 4.f * g.invDx * g.dx;
                        const float fx[3] = {st.fx.x, st.fx.y, st.fx.z};
                        const float Svv[3] = {Sv.x, Sv.y, Sv.z};
#pragma unroll
                        for (int r = 0; r < 3; ++r)
#pragma unroll
                            for (int c = 0; c < 3; ++c)
                                Cn.m[3 * c + r] = s4 * (T[3 * r + c] - fx[r] * Svv[c]);
                    }
                    V3 xn = x + Sv * p.dt;
                    xn = v3(fminf(fmaxf(xn.x, g.gmin.x), g.gmax.x), fminf(fmaxf(xn.y, g.gmin.y), g.gmax.y),
                            fminf(fmaxf(xn.z, g.gmin.z), g.gmax.z));
                    V3 vn = Sv;
                    if (p.numShapes > 0)
                    {
                        int bx0, by0, bz0;
                        const unsigned blk = baseBlock(g, st, bx0, by0, bz0);
                        const bool near = blockRegion(g, bx0, by0, bz0).contains(xn);
                        CoupleAtomic noCouple{nullptr, nullptr}; // particle push-out exchanges no momentum
                        rigidContact<true>(vn, x4.w, xn, shp, p.numShapes, sdf, false, noCouple,
                                           near ? blockShapeMask[blk] : ~0ull);
                    }
                    M3 Mu;
#pragma unroll
                    for (int e = 0; e < 9; ++e)
                        Mu.m[e] = ((e % 4) == 0 ? 1.f : 0.f) + Cn.m[e] * p.dt;
                    Fp = matmul(Mu, Fp);
                    if (!(isfinite(xn.x) && isfinite(xn.y) && isfinite(xn.z) && isfinite(vn.x) && isfinite(vn.y) &&
                          isfinite(vn.z)))
                        atomicOr(&hdr->status, CRB200_STATUS_NAN_STATE);
                    if (Export)
                    {
                        // the last substep of a call: positions and velocities to the caller, C for
                        // the next call's first P2G and for readback
                        callerX[id] = make_float4(xn.x, xn.y, xn.z, x4.w);
                        callerV[id] = make_float4(vn.x, vn.y, vn.z, 0.f);
                        storeM3(rs.C, rs.stride, s, Cn);
                    }
                    else
                    {
                        rs.x[s] = make_float4(xn.x, xn.y, xn.z, x4.w);
                        if (slicers)
                            rs.v[s] = make_float4(vn.x, vn.y, vn.z, 0.f);
                    }
                    storeM3(rs.F, rs.stride, s, Fp);
                    x = xn;
                    v = vn;
                    Cp = Cn;
                }
                if (DoP2G)
                {
                    const float4 mp = mixed ? rs.mat[s] : matU;
                    RawParticle raw;
                    raw.x4 = make_float4(x.x, x.y, x.z, x4.w);
                    raw.v4 = make_float4(v.x, v.y, v.z, 0.f);
                    raw.mp = mp;
                    raw.mt = __float_as_int(mp.z);
#pragma unroll
                    for (int e = 0; e < 9; ++e)
                    {
                        raw.F[e] = Fp.m[e];
                        raw.C[e] = Cp.m[e];
                    }
                    raw.v0 = V0p;
                    const Stencil sn = stencilOf(g, x);
                    bool ood = !sn.finite;
                    if (sn.finite)
                        (void)cellKey(g, sn, &ood);
                    if (ood)
                        atomicOr(&hdr->status, CRB200_STATUS_OUT_OF_DOMAIN);
                    unsigned msk = 0u;
                    if (slicers)
                    {
                        msk = sn.finite ? cutMaskOf(g, x, sn, shp, p.numShapes, sdf) : 0u;
                        rs.cut[s] = msk;
                    }
                    float rec[kRec];
                    // false: non-finite, or a base cell outside [0, n-2] (then nothing was scattered)
                    const bool inside = buildRecord<0>(p, id, raw, nullptr, rs.stride, msk, false, nullptr, nullptr,
                                                       nullptr, rec);
                    // The particle's current cell, when it lies in this block: the cell's threads sum
                    // its record, at a rank taken from the cell's shared counter (one atomic per group
                    // of lanes in the same cell).  Particles that left the block, or beyond a cell's
                    // kResRanks, are added by atomics.
                    const int qx = sn.b[0] - 4 * bx, qy = sn.b[1] - 4 * by, qz = sn.b[2] - 4 * bz;
                    const bool inBlock = inside && msk == 0u && qx >= 0 && qx <= 3 && qy >= 0 && qy <= 3 && qz >= 0 &&
                                         qz <= 3;
                    unsigned rank = (unsigned)kResRanks;
                    if (inBlock)
                    {
                        const int c = qx + 4 * (qy + 4 * qz);
                        const unsigned am = __activemask(), lane = threadIdx.x & 31u;
                        const unsigned peers = __match_any_sync(am, c);
                        const int leader = __ffs(peers) - 1;
                        unsigned base = 0u;
                        if ((int)lane == leader)
                            base = atomicAdd(&S.count[c], (unsigned)__popc(peers));
                        base = __shfl_sync(peers, base, leader);
                        rank = base + (unsigned)__popc(peers & ((1u << lane) - 1u));
                        if (rank < (unsigned)kResRanks)
                        {
                            const int q = (int)rank * kResRecStride + c;
#pragma unroll
                            for (int e = 0; e < kRec; ++e)
                                S.rec[e][q] = rec[e];
                        }
                    }
                    if (rank >= (unsigned)kResRanks)
                    {
                        const int rx = sn.b[0] - ox, ry = sn.b[1] - oy, rz = sn.b[2] - oz;
                        if (inBlock)
                        {
                            // a crowded cell: the cell's first kResRanks records cover the same nodes,
                            // so the window flush lists their blocks
                            resScatterRed(g, sn, rec, 0u, gridA);
                        }
                        else if (inside && rx >= 0 && rx <= 5 && ry >= 0 && ry <= 5 && rz >= 0 && rz <= 5)
                        {
                            // left the block, not the window: the blocks of its stencil (within the
                            // 3x3x3 neighbourhood of this block) are listed by the flush
                            resScatterRed(g, sn, rec, msk, gridA);
                            unsigned bits = 0u;
                            const int l0[3] = {(sn.b[0] >> 2) - bx + 1, (sn.b[1] >> 2) - by + 1, (sn.b[2] >> 2) - bz + 1};
                            const int l1[3] = {(min(sn.b[0] + 2, g.n.x - 1) >> 2) - bx + 1,
                                               (min(sn.b[1] + 2, g.n.y - 1) >> 2) - by + 1,
                                               (min(sn.b[2] + 2, g.n.z - 1) >> 2) - bz + 1};
                            for (int zz = l0[2]; zz <= l1[2]; ++zz)
                                for (int yy = l0[1]; yy <= l1[1]; ++yy)
                                    for (int xx = l0[0]; xx <= l1[0]; ++xx)
                                        bits |= 1u << (xx + 3 * yy + 9 * zz);
                            atomicOr(&S.touchedBits, bits);
                        }
                        else if (sn.finite)
                        {
                            // left the window, or a stencil across the grid boundary (the record is
                            // complete either way; only a non-finite position leaves it empty)
                            RecVal rv;
#pragma unroll
                            for (int e = 0; e < kRec; ++e)
                                rv.r[e] = rec[e];
                            resScatterGlobal(g, sn, rv, msk, gridA, touchedFlag, touchedList, hdr);
                            atomicAdd(&S.outside, 1u);
                        }
                        if (!inBlock)
                            atomicAdd(&S.movers, 1u);
                    }
                }
            }
            if (!DoP2G)
                continue;
            __syncthreads();
            // ---- records by cell: thread (cell c, x-slab sl) over the cell's first kResRanks particles
            {
                const int c = tid & 63, sl = tid >> 6;
                const float slf = (float)sl;
                const unsigned cnt = min(S.count[c], (unsigned)kResRanks);
                float acc[3][3][4];
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int k = 0; k < 3; ++k)
#pragma unroll
                        for (int ch = 0; ch < 4; ++ch)
                            acc[j][k][ch] = 0.f;
                for (unsigned r = 0; r < cnt; ++r)
                {
                    const int q = (int)r * kResRecStride + c;
                    float rc[kRec];
#pragma unroll
                    for (int e = 0; e < kRec; ++e)
                        rc[e] = S.rec[e][q];
                    float w[3][3];
                    weights(v3(rc[13], rc[14], rc[15]), w);
                    const float wx = sl == 0 ? w[0][0] : (sl == 1 ? w[1][0] : w[2][0]);
                    const V3 ui = fma3(v3(rc[4], rc[5], rc[6]), slf, v3(rc[0], rc[1], rc[2]));
                    const V3 a1 = v3(rc[7], rc[8], rc[9]), a2 = v3(rc[10], rc[11], rc[12]);
#pragma unroll
                    for (int j = 0; j < 3; ++j)
                    {
                        const V3 uij = j == 0 ? ui : fma3(a1, (float)j, ui);
                        const float wij = wx * w[j][1];
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                            fma4acc(acc[j][k], k == 0 ? uij : fma3(a2, (float)k, uij), rc[3], wij * w[k][2]);
                    }
                }
                // Shared-memory float reductions into the output window.  For one offset (j, k) the
                // 32 cells of a warp add to 32 distinct nodes in 32 distinct banks (z stride
                // kOutZ), so a warp's reductions never collide with each other; neighbouring cells
                // of other warps share nodes, which the reductions resolve in hardware.
                if (cnt)
                {
                    const int cx = c & 3, cy = (c >> 2) & 3, cz = c >> 4;
#pragma unroll
                    for (int j = 0; j < 3; ++j)
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                        {
                            const int t = (cx + 1 + sl) + 8 * (cy + 1 + j) + kOutZ * (cz + 1 + k);
#pragma unroll
                            for (int ch = 0; ch < 4; ++ch)
                                atomicAdd(&S.out[ch][t], acc[j][k][ch]);
                        }
                }
            }
            __syncthreads();
            // ---- the output window into the accumulation grid
            unsigned bits = 0u;
            for (int t = tid; t < kWinNodes; t += kResThreads)
            {
                const int tx = t & 7, ty = (t >> 3) & 7, tz = t >> 6;
                const int o = tx + 8 * ty + kOutZ * tz;
                const float px = S.out[0][o], py = S.out[1][o], pz = S.out[2][o], m = S.out[3][o];
                S.out[0][o] = 0.f;
                S.out[1][o] = 0.f;
                S.out[2][o] = 0.f;
                S.out[3][o] = 0.f;
                if (px == 0.f && py == 0.f && pz == 0.f && m == 0.f)
                    continue;
                const int i = ox + tx, j = oy + ty, k = oz + tz;
                if (!inGrid(g, i, j, k))
                    continue;
                atomicAdd(&gridA[nodeAddr(g, i, j, k)], make_float4(px, py, pz, m));
                bits |= 1u << (((i >> 2) - bx + 1) + 3 * ((j >> 2) - by + 1) + 9 * ((k >> 2) - bz + 1));
            }
            bits = __reduce_or_sync(0xffffffffu, bits);
            if ((tid & 31) == 0 && bits)
                atomicOr(&S.touchedBits, bits);
            __syncthreads();
            if (tid < 64)
                S.count[tid] = 0u; // read by the accumulation above, before the last barrier
            if (tid < 27 && ((S.touchedBits >> tid) & 1u))
            {
                const int nx = bx - 1 + tid % 3, ny = by - 1 + (tid / 3) % 3, nz = bz - 1 + tid / 9;
                markTouched(g.blockBase + (unsigned)(nx + g.nb.x * (ny + g.nb.y * nz)), touchedFlag, touchedList, hdr);
            }
        }
        if (DoP2G)
        {
            __syncthreads();
            if (tid == 0)
            {
                if (S.movers)
                    atomicAdd(&hdr->resMovers, S.movers);
                if (S.outside)
                    atomicAdd(&hdr->resOutside, S.outside);
            }
        }
    }

    // Whether this call re-sorts the resident slots: on request of the host (first call, changed
    // particle set or state) or when the previous call left particles outside their block's window
    // or more than one in 64 outside its block.  The sort kernels return at once otherwise.
    __global__ void k_resDecide(SortHeader *hdr)
    {
        const bool want = hdr->resForce != 0u || hdr->resOutside != 0u ||
                          (unsigned long long)hdr->resMovers * 64ull > (unsigned long long)hdr->numSorted;
        hdr->sortSkip = want ? 0u : 1u;
        hdr->resOutside = 0u;
        if (want)
            hdr->matMixed = 0u;
    }

    // After a re-sort: the new slot order's particle state into the scratch arrays.  Positions and
    // materials come from the caller's buffers (velocities are read from there by the call's first
    // P2G); F, C and V0 from the particle-id planes (resFromPlanes) or from the particle's previous
    // resident slot.
    __global__ void k_resGather(const SortHeader *hdr, const unsigned *__restrict__ sortedIds,
                                const float4 *__restrict__ callerX, const float4 *__restrict__ callerV,
                                const float4 *__restrict__ matParams, const int *__restrict__ matType,
                                const float *__restrict__ Fid, const float *__restrict__ Cid,
                                const float *__restrict__ V0id, ResState rs, const unsigned *__restrict__ slotOf,
                                float4 *__restrict__ x2, float *__restrict__ V02, float *__restrict__ F2,
                                float *__restrict__ C2, float4 *__restrict__ mat2, unsigned *__restrict__ id2,
                                SortHeader *hdrw)
    {
        if (hdr->sortSkip)
            return;
        const unsigned n = hdr->numSorted, stride = rs.stride;
        const bool fromPlanes = hdr->resFromPlanes != 0u;
        const unsigned id0 = n ? sortedIds[0] : 0u;
        const float4 m0 = n ? matParams[id0] : make_float4(0.f, 0.f, 0.f, 0.f);
        const int t0 = n ? matType[id0] : 0;
        bool mixed = false;
        for (unsigned s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
        {
            const unsigned id = sortedIds[s];
            const float4 x4 = callerX[id], mp = matParams[id];
            const int mt = matType[id];
            float v0;
            // a particle without a previous slot (slotOf is cleared to ~0 when the arrays are made)
            // takes its F, C and V0 from the planes even when the rest comes from the slots
            const unsigned o = fromPlanes ? 0xFFFFFFFFu : slotOf[id];
            if (o >= stride)
            {
#pragma unroll
                for (int k = 0; k < 9; ++k)
                {
                    F2[k * stride + s] = Fid[k * stride + id];
                    C2[k * stride + s] = Cid[k * stride + id];
                }
                v0 = V0id[id];
            }
            else
            {
#pragma unroll
                for (int k = 0; k < 9; ++k)
                {
                    F2[k * stride + s] = rs.F[k * stride + o];
                    C2[k * stride + s] = rs.C[k * stride + o];
                }
                v0 = rs.V0[o];
            }
            x2[s] = x4;
            V02[s] = v0;
            mat2[s] = make_float4(mp.x, mp.y, __int_as_float(mt), 0.f);
            id2[s] = id;
            mixed |= __float_as_uint(mp.x) != __float_as_uint(m0.x) || __float_as_uint(mp.y) != __float_as_uint(m0.y) ||
                     mt != t0;
        }
        if (__any_sync(0xffffffffu, mixed) && (threadIdx.x & 31) == 0)
            atomicOr(&hdrw->matMixed, 1u);
        if (blockIdx.x == 0 && threadIdx.x == 0)
            hdrw->matUniform = make_float4(m0.x, m0.y, __int_as_float(t0), 0.f);
    }

    // The scratch arrays become the resident state; each particle's slot is recorded.
    __global__ void k_resCopyBack(SortHeader *hdr, ResState rs, unsigned *__restrict__ slotOf,
                                  const float4 *__restrict__ x2, const float *__restrict__ V02,
                                  const float *__restrict__ F2, const float *__restrict__ C2,
                                  const float4 *__restrict__ mat2, const unsigned *__restrict__ id2,
                                  float4 *__restrict__ matOut, unsigned *__restrict__ idOut)
    {
        if (hdr->sortSkip)
            return;
        const unsigned n = hdr->numSorted, stride = rs.stride;
        for (unsigned s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
        {
            rs.x[s] = x2[s];
            rs.V0[s] = V02[s];
#pragma unroll
            for (int k = 0; k < 9; ++k)
            {
                rs.F[k * stride + s] = F2[k * stride + s];
                rs.C[k * stride + s] = C2[k * stride + s];
            }
            matOut[s] = mat2[s];
            const unsigned id = id2[s];
            idOut[s] = id;
            slotOf[id] = s;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0)
        {
            hdr->resForce = 0u;
            hdr->resFromPlanes = 0u;
        }
    }

    // Resident F and C (or, when `cutOut` is given, the cut masks) back to the particle-id order.
    __global__ void k_resExport(const SortHeader *__restrict__ hdr, ResState rs, float *__restrict__ Fid,
                                float *__restrict__ Cid, unsigned *__restrict__ cutOut)
    {
        const unsigned n = hdr->numSorted, stride = rs.stride;
        for (unsigned s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
        {
            const unsigned id = rs.id[s];
            if (cutOut)
            {
                cutOut[id] = rs.cut[s];
                continue;
            }
#pragma unroll
            for (int k = 0; k < 9; ++k)
            {
                Fid[k * stride + id] = rs.F[k * stride + s];
                Cid[k * stride + id] = rs.C[k * stride + s];
            }
        }
    }
} // namespace crb200
