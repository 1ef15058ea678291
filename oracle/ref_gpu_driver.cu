// ORACLE / TEST INFRASTRUCTURE ONLY: the reference's own CUDA solvers (GpuMlsMpmSolver,
// GpuPbMpmSolver, GpuStandardMpmSolver from src/solver/gpu_*_mpm_solver.cu, compiled for sm_100a
// by `make -C oracle ref-gpu` from the sources where they lie) driven through their MpmSolver
// interface the way SimulationFactoryImpl::createScene and SceneImpl drive them
// (src/engine/simulation_factory_impl.cpp:296-349, src/engine/scene_impl.cpp:42-93, 202-220,
// 308-330).  Used for GPU-vs-GPU parity and to time the reference's GPU solver on the same B200.
//
//     ref_gpu_driver scene.bin warmup steps out.bin
//
// scene.bin (little endian, written by oracle_py.write_gpu_scene):
//   int32 n, solverType, iterations, contactModel; float32 cell, dt, gmin[3], gmax[3], gravity[3];
//   float32 positionMass[4n], velocity[4n], params0[4n]; int32 type[n]; uint8 mask[n];
//   int32 S (all shapes); int32 shapeType[S], geometryIdx[S]; float32 position, rotation, invScale,
//   linearVelocity, angularVelocity, comInvMass, inertiaInv0, inertiaInv1, params0 [S x 4 each];
//   int32 K (shapes in the scene); int32 shapeIds[K]; int32 G; int32 geometryType[G];
//   float32 geometryParams[G x 4]; int32 D; int32 dims[D x 4]; float32 lowerBoundCellSize[D x 4];
//   int32 M; float32 sdfData[M x 4].
// Scenes with analytic geometries only (no triangle-mesh or line-segment SDF data).
// Runs `warmup` substeps, then `steps` substeps timed with CUDA events on the solver stream, and
// writes positionMass[4n], velocity[4n] and force, torque [S x 4] to out.bin; prints the mean
// milliseconds per timed substep.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "gpu_mls_mpm_solver.cuh"
#include "gpu_pb_mpm_solver.cuh"
#include "gpu_standard_mpm_solver.cuh"

using namespace crmpm;

namespace
{
    FILE *gIn = nullptr;
    bool gOk = true;

    template <class T> std::vector<T> readVec(size_t count)
    {
        std::vector<T> v(count);
        if (count && std::fread(v.data(), sizeof(T), count, gIn) != count)
            gOk = false;
        return v;
    }

    // a count from the file; a negative or absurd one marks the file bad and reads as 0
    int readCount()
    {
        const auto c = readVec<int>(1);
        if (!gOk || c[0] < 0 || c[0] > (1 << 28))
        {
            gOk = false;
            return 0;
        }
        return c[0];
    }

    template <class T> T *upload(const std::vector<T> &h, size_t minCount = 1)
    {
        T *d = nullptr;
        const size_t count = h.size() < minCount ? minCount : h.size();
        cudaMalloc(&d, count * sizeof(T));
        cudaMemset(d, 0, count * sizeof(T));
        if (!h.empty())
            cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
        return d;
    }
} // namespace

int main(int argc, char **argv)
{
    if (argc < 5)
        return 2;
    gIn = std::fopen(argv[1], "rb");
    if (!gIn)
        return 2;
    const auto hi = readVec<int>(4);
    const auto hf = readVec<float>(11);
    if (!gOk || hi[0] <= 0 || hi[0] > (1 << 28))
        return 2;
    const int n = hi[0], type = hi[1], iterations = hi[2], contactModel = hi[3];
    const auto pm = readVec<float4>(n), vel = readVec<float4>(n), mp = readVec<float4>(n);
    const auto mt = readVec<int>(n);
    const auto mask = readVec<unsigned char>(n);
    const int ns = readCount();
    const auto stype = readVec<int>(ns), sgeom = readVec<int>(ns);
    std::vector<std::vector<float4>> sf;
    for (int k = 0; k < 9; ++k)
        sf.push_back(readVec<float4>(ns));
    const int nk = readCount();
    const auto sids = readVec<int>(nk);
    const int ng = readCount();
    const auto gtype = readVec<int>(ng);
    const auto gparams = readVec<float4>(ng);
    const int nsdf = readCount();
    const auto sdims = readVec<int4>(nsdf);
    const auto slbcs = readVec<float4>(nsdf);
    const int sdfLen = readCount();
    const auto sdata = readVec<float4>(sdfLen);
    std::fclose(gIn);
    if (!gOk || nk > ns || nsdf < 1 || sdfLen < 1)
        return 2;
    for (int k = 0; k < nk; ++k)
        if (sids[k] < 0 || sids[k] >= ns)
            return 2;
    for (int k = 0; k < ns; ++k)
        if (sgeom[k] < 0 || sgeom[k] >= ng)
            return 2;
    // analytic geometries only (box, sphere, plane, capsule, quad slicer, arc): the SDF-backed ones
    // index the SDF arrays through offsets this driver does not check
    for (int k = 0; k < ng; ++k)
        if (gtype[k] < 0 || gtype[k] > 8 || gtype[k] == 4 || gtype[k] == 6 || gtype[k] == 7)
            return 2;
    const int warmup = std::atoi(argv[2]), steps = std::atoi(argv[3]);

    ParticleData pd(n);
    pd.positionMass = upload(pm);
    pd.velocity = reinterpret_cast<Vec3f *>(upload(vel));
    ParticleMaterialData md(n);
    md.params0 = upload(mp);
    md.type = reinterpret_cast<ParticleMaterialType *>(upload(mt));
    unsigned char *dMask = upload(mask);
    std::vector<unsigned> idx;
    for (int i = 0; i < n; ++i)
        if (mask[i])
            idx.push_back((unsigned)i);
    unsigned *dIdx = upload(idx);

    ShapeData sd;
    sd.type = reinterpret_cast<ShapeType *>(upload(stype));
    sd.geometryIdx = upload(sgeom);
    sd.position = reinterpret_cast<Vec3f *>(upload(sf[0]));
    sd.rotation = reinterpret_cast<Quat *>(upload(sf[1]));
    sd.invScale = reinterpret_cast<Vec3f *>(upload(sf[2]));
    sd.linearVelocity = reinterpret_cast<Vec3f *>(upload(sf[3]));
    sd.angularVelocity = reinterpret_cast<Vec3f *>(upload(sf[4]));
    sd.comInvMass = upload(sf[5]);
    sd.inertiaInv0 = upload(sf[6]);
    sd.inertiaInv1 = upload(sf[7]);
    sd.params0 = upload(sf[8]);
    sd.force = upload(std::vector<float4>(ns > 0 ? ns : 1, make_float4(0.f, 0.f, 0.f, 0.f)));
    sd.torque = upload(std::vector<float4>(ns > 0 ? ns : 1, make_float4(0.f, 0.f, 0.f, 0.f)));
    sd.size = ns;
    GeometryData gd;
    gd.type = reinterpret_cast<GeometryType *>(upload(gtype));
    gd.params0 = upload(gparams);
    gd.size = ng;
    GeometrySdfData sdf;
    sdf.dimemsion = reinterpret_cast<Vec3i *>(upload(sdims));
    sdf.lowerBoundCellSize = upload(slbcs);
    sdf.gradientSignedDistance = upload(sdata);
    int *dIds = upload(sids);

    const float cell = hf[0], dt = hf[1];
    Bounds3 bounds(Vec3f(hf[2], hf[3], hf[4]), Vec3f(hf[5], hf[6], hf[7]));
    MpmSolverGpu *solver = nullptr;
    if (type == 1)
        solver = new GpuMlsMpmSolver(n, cell, bounds);
    else if (type == 3)
        solver = new GpuPbMpmSolver(n, cell, bounds);
    else if (type == 5)
        solver = new GpuStandardMpmSolver(n, cell, bounds);
    else
        return 2;
    cudaStream_t stream;
    cudaStreamCreate(&stream);
    solver->setCudaStream(stream);
    solver->bindParticleData(pd);
    solver->bindParticleMaterials(md);
    solver->bindActiveMask(dMask);
    solver->setGravity(Vec3f(hf[8], hf[9], hf[10]));
    solver->setIntegrationStepSize(dt);
    solver->setSolverIterations(iterations);
    solver->setNumActiveParticles((unsigned)n);
    solver->setNumShapes(nk);
    solver->bindShapeIds(dIds);
    solver->bindShapeData(sd);
    solver->bindGeometryData(gd);
    solver->bindGeometrySdfData(sdf);
    solver->setShapeContactModel(static_cast<ShapeContactModel>(contactModel));
    solver->initialize();
    solver->computeInitialData((unsigned)idx.size(), dIdx);
    for (int s = 0; s < warmup; ++s)
        solver->step();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, stream);
    for (int s = 0; s < steps; ++s)
        solver->step();
    cudaEventRecord(e1, stream);
    solver->fetchResults();
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    std::vector<float4> x(n), v(n), f(ns > 0 ? ns : 1), t(ns > 0 ? ns : 1);
    cudaMemcpy(x.data(), pd.positionMass, 16ull * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(v.data(), pd.velocity, 16ull * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(f.data(), sd.force, 16ull * f.size(), cudaMemcpyDeviceToHost);
    cudaMemcpy(t.data(), sd.torque, 16ull * t.size(), cudaMemcpyDeviceToHost);
    solver->release();
    FILE *o = std::fopen(argv[4], "wb");
    if (!o)
        return 2;
    std::fwrite(x.data(), 16, n, o);
    std::fwrite(v.data(), 16, n, o);
    std::fwrite(f.data(), 16, ns, o);
    std::fwrite(t.data(), 16, ns, o);
    std::fclose(o);
    const cudaError_t err = cudaGetLastError();
    std::printf("ms_per_substep %.6f steps %d particles %d cuda %s\n", steps > 0 ? ms / steps : 0.0, steps, n,
                cudaGetErrorString(err));
    return err == cudaSuccess ? 0 : 1;
}
