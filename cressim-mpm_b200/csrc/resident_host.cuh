// Host side of the resident single-scene MLS path (kernels in resident.cuh; included at the end of
// mpm_kernels.cu).
//
// A call of n substeps is three pieces:
//   start   shape gather; the re-sort decision; the sort chain, gather and copy-back (all of which
//           return at once when no re-sort is due); P2G of substep 0 from the caller's positions
//   middle  (n - 1 times) grid update of substep k; the fused G2P of k and P2G of k + 1
//   last    grid update of substep n - 1; G2P that writes positions and velocities to the caller's
//           buffers
// With a stream each piece is replayed from its own CUDA graph.  After the call the caller's
// positions and velocities are current, as with the particle-id-ordered path; F and C are current
// in the resident slots and are written back to the particle-id planes whenever something reads
// or replaces those (residentSyncPlanes).
#pragma once

namespace crb200
{
    bool Solver::residentUsable() const
    {
        return residentOn && initialized && !isBatch() && solverType == CRB200_SOLVER_GPU_MLS && !detP2G &&
               !detCoupling && tapeActive < 0 && !adjReplay && outX == nullptr && numShapes <= kMaxShapes;
    }

    int Solver::residentAlloc()
    {
        if (res.x)
            return CRB200_OK;
        const size_t n = (size_t)numMaxParticles;
        float4 *mat = nullptr;
        unsigned *id = nullptr;
        CRB_CHECK(cudaMalloc(&res.x, n * sizeof(float4)));
        CRB_CHECK(cudaMalloc(&res.v, n * sizeof(float4)));
        CRB_CHECK(cudaMalloc(&res.V0, n * sizeof(float)));
        CRB_CHECK(cudaMalloc(&res.F, 9 * n * sizeof(float)));
        CRB_CHECK(cudaMalloc(&res.C, 9 * n * sizeof(float)));
        CRB_CHECK(cudaMalloc(&mat, n * sizeof(float4)));
        CRB_CHECK(cudaMalloc(&id, n * sizeof(unsigned)));
        CRB_CHECK(cudaMalloc(&res.cut, n * sizeof(unsigned)));
        res.mat = mat;
        res.id = id;
        res.stride = (unsigned)n;
        CRB_CHECK(cudaMalloc(&resSlotOf, n * sizeof(unsigned)));
        CRB_CHECK(cudaMalloc(&resX2, n * sizeof(float4)));
        CRB_CHECK(cudaMalloc(&resV02, n * sizeof(float)));
        CRB_CHECK(cudaMalloc(&resMat2, n * sizeof(float4)));
        CRB_CHECK(cudaMalloc(&resF2, 9 * n * sizeof(float)));
        CRB_CHECK(cudaMalloc(&resC2, 9 * n * sizeof(float)));
        CRB_CHECK(cudaMalloc(&resId2, n * sizeof(unsigned)));
        CRB_CHECK(cudaMalloc(&touchedFlag, (size_t)totalBlocks * sizeof(unsigned)));
        CRB_CHECK(cudaMemsetAsync(res.cut, 0, n * sizeof(unsigned), stream));
        CRB_CHECK(cudaMemsetAsync(resSlotOf, 0xff, n * sizeof(unsigned), stream));
        CRB_CHECK(cudaMemsetAsync(touchedFlag, 0, (size_t)totalBlocks * sizeof(unsigned), stream));
        const int maxSmem = (int)(sizeof(ResShared) + kMaxShapes * sizeof(ShapeRec));
        CRB_CHECK(cudaFuncSetAttribute(k_g2p2g<false, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxSmem));
        CRB_CHECK(cudaFuncSetAttribute(k_g2p2g<true, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxSmem));
        CRB_CHECK(cudaFuncSetAttribute(k_g2p2g<true, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxSmem));
        resValid = false;
        resPlanesStale = false;
        return CRB200_OK;
    }

    int Solver::residentSyncPlanes()
    {
        if (!resValid || !resPlanesStale)
            return CRB200_OK;
        k_resExport<<<strideCtas, 256, 0, stream>>>(header, res, F, Cm, nullptr);
        CRB_LAUNCHED(1);
        resPlanesStale = false;
        return CRB200_OK;
    }

    // Back to the particle-id order: F and C to the planes, the resident state dropped, and the
    // sort kernels no longer told to skip (the particle-id path sorts every substep).
    int Solver::residentRetire()
    {
        if (int r = residentSyncPlanes())
            return r;
        if (resValid)
            CRB_CHECK(cudaMemsetAsync(&header->sortSkip, 0, sizeof(unsigned), stream));
        resValid = false;
        return CRB200_OK;
    }

    int Solver::copyCutMasks(unsigned *out)
    {
        const unsigned n = totalParticles();
        CRB_CHECK(cudaMemsetAsync(out, 0, n * sizeof(unsigned), stream));
        k_resExport<<<strideCtas, 256, 0, stream>>>(header, res, nullptr, nullptr, out);
        CRB_LAUNCHED(1);
        return CRB200_OK;
    }

    // One piece of a resident call (see the file comment).  With phase timing on, every launch is
    // bracketed by events and waited for: phase 0 the call start up to its P2G, 1 the P2G and the
    // fused kernels, 2 the grid updates, 3 the last G2P.
    int Solver::residentPiece(int which)
    {
        const StepParams p = params();
        const SceneTable sc = sceneTable();
        const SdfPtrs sp{reinterpret_cast<const int4 *>(sdf.dimension), reinterpret_cast<const float4 *>(sdf.lowerBoundCellSize),
                         reinterpret_cast<const float4 *>(sdf.gradientSignedDistance)};
        float4 *cf = reinterpret_cast<float4 *>(shapes.force), *ct = reinterpret_cast<float4 *>(shapes.torque);
        if (scratchCoupling)
        {
            cf = adjForce;
            ct = adjTorque;
        }
        const size_t smem = sizeof(ResShared) + (size_t)numShapes * sizeof(ShapeRec);
        cudaEvent_t t0 = phaseEv[0], t1 = phaseEv[1];
        auto begin = [&]() -> int {
            if (phaseTiming)
                CRB_CHECK(cudaEventRecord(t0, stream));
            return CRB200_OK;
        };
        auto end = [&](int phase, bool fused) -> int {
            if (!phaseTiming)
                return CRB200_OK;
            CRB_CHECK(cudaEventRecord(t1, stream));
            CRB_CHECK(cudaEventSynchronize(t1));
            float ms = 0.f;
            CRB_CHECK(cudaEventElapsedTime(&ms, t0, t1));
            phaseMs[phase] += ms;
            if (fused)
            {
                fusedMs += ms;
                fusedLaunches++;
            }
            return CRB200_OK;
        };
        auto clearCounts = [&]() -> int {
            // numTouchedBlocks, resMovers, touchedNodes
            CRB_CHECK(cudaMemsetAsync(&header->numTouchedBlocks, 0, 3 * sizeof(unsigned), stream));
            return CRB200_OK;
        };
        int r = CRB200_OK;
        if (which == 0)
        {
            if ((r = begin()) != CRB200_OK)
                return r;
            if (numShapes > 0)
            {
                gatherShapes(stream);
                CRB_LAUNCHED(1);
            }
            k_resDecide<<<1, 1, 0, stream>>>(header);
            CRB_LAUNCHED(1);
            if ((r = sortParticles(p, false)) != CRB200_OK)
                return r;
            k_resGather<<<strideCtas, 256, 0, stream>>>(header, sortedIds, positionMass, velocity, matParams, matType, F,
                                                         Cm, V0, res, resSlotOf, resX2, resV02, resF2, resC2, resMat2,
                                                         resId2, header);
            k_resCopyBack<<<strideCtas, 256, 0, stream>>>(header, res, resSlotOf, resX2, resV02, resF2, resC2, resMat2,
                                                           resId2, const_cast<float4 *>(res.mat),
                                                           const_cast<unsigned *>(res.id));
            CRB_LAUNCHED(2);
            if ((r = clearCounts()) != CRB200_OK || (r = end(0, false)) != CRB200_OK || (r = begin()) != CRB200_OK)
                return r;
            k_g2p2g<false, true, false><<<resCtas, kResThreads, smem, stream>>>(
                p, header, activeList, blockStart, res, positionMass, velocity, gridV, gridA, touchedFlag, touchedList,
                shapeTable, sp, blockShapeMask, sc.flags);
            CRB_LAUNCHED(1);
            return end(1, false);
        }
        if ((r = begin()) != CRB200_OK)
            return r;
        k_gridUpdate<false, 0><<<updCtas, 256, 0, stream>>>(p, sc, header, touchedList, shapeTable, sp, gridA, gridF,
                                                             gridV, cf, ct, true, blockShapeMask, nullptr, nullptr,
                                                             nullptr, nullptr, 0u, nullptr, nullptr, blockFlags,
                                                             touchedFlag);
        CRB_LAUNCHED(1);
        if ((r = end(2, false)) != CRB200_OK)
            return r;
        if (which == 1)
        {
            if ((r = clearCounts()) != CRB200_OK || (r = begin()) != CRB200_OK)
                return r;
            k_g2p2g<true, true, false><<<resCtas, kResThreads, smem, stream>>>(
                p, header, activeList, blockStart, res, positionMass, velocity, gridV, gridA, touchedFlag, touchedList,
                shapeTable, sp, blockShapeMask, sc.flags);
            CRB_LAUNCHED(1);
            return end(1, true);
        }
        if ((r = begin()) != CRB200_OK)
            return r;
        k_g2p2g<true, false, true><<<resCtas, kResThreads, smem, stream>>>(
            p, header, activeList, blockStart, res, positionMass, velocity, gridV, gridA, touchedFlag, touchedList,
            shapeTable, sp, blockShapeMask, sc.flags);
        CRB_LAUNCHED(1);
        return end(3, false);
    }

    int Solver::residentStep(int n)
    {
        if (numActive > 0 && (!matParams || !matType || !activeMask))
        {
            setLastError("step: particle materials or active mask not bound");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        if (numShapes > 0 && (!shapeIds || !shapes.type || !geometries.type))
        {
            setLastError("step: shapes are enabled but shape ids / shape data / geometry data are not bound");
            return CRB200_ERR_NOT_INITIALIZED;
        }
        if (int r = residentAlloc())
            return r;
        if (resCtas == 0 || resGraphVersion != configVersion)
        {
            // CTAs of the fused kernel: its occupancy at this shape count, times the SMs (and the
            // autotuned multiple)
            int dev = 0, sms = 0, perSm = 0;
            CRB_CHECK(cudaGetDevice(&dev));
            CRB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            CRB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &perSm, k_g2p2g<true, true, false>, kResThreads, sizeof(ResShared) + (size_t)numShapes * sizeof(ShapeRec)));
            resCtas = sms * std::max(perSm, 1) * std::max(resMult, 1);
        }
        if (!resValid)
        {
            // re-sort at this call, F, C and V0 from the particle-id planes (resForce, resFromPlanes)
            CRB_CHECK(cudaMemsetAsync(&header->resForce, 1, 2 * sizeof(unsigned), stream));
            resValid = true;
        }
        int r = invalidateRecords();
        if (r != CRB200_OK)
            return r;
        if (stream == nullptr || phaseTiming)
        {
            if (phaseTiming)
                for (int k = 0; k < 2; ++k)
                    if (!phaseEv[k])
                        CRB_CHECK(cudaEventCreate(&phaseEv[k]));
            if ((r = residentPiece(0)) != CRB200_OK)
                return r;
            for (int k = 1; k < n; ++k)
                if ((r = residentPiece(1)) != CRB200_OK)
                    return r;
            if ((r = residentPiece(2)) != CRB200_OK)
                return r;
            if (phaseTiming)
                phaseSteps += n;
            resPlanesStale = true;
            return CRB200_OK;
        }
        if (resGraphVersion != configVersion)
        {
            for (int k = 0; k < 3; ++k)
            {
                if (resGraph[k])
                {
                    cudaGraphExecDestroy(resGraph[k]);
                    resGraph[k] = nullptr;
                }
                const uint64_t before = launchCount();
                CRB_CHECK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
                r = residentPiece(k);
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
                e = cudaGraphInstantiate(&resGraph[k], g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess)
                    return cudaFail(e, "cudaGraphInstantiate");
                resGraphKernels[k] = (int)captured;
            }
            resGraphVersion = configVersion;
        }
        CRB_CHECK(cudaGraphLaunch(resGraph[0], stream));
        for (int k = 1; k < n; ++k)
            CRB_CHECK(cudaGraphLaunch(resGraph[1], stream));
        CRB_CHECK(cudaGraphLaunch(resGraph[2], stream));
        noteLaunches((uint64_t)resGraphKernels[0] + (uint64_t)resGraphKernels[1] * (uint64_t)(n - 1) +
                     (uint64_t)resGraphKernels[2]);
        resPlanesStale = true;
        return CRB200_OK;
    }
} // namespace crb200
