// ORACLE / TEST INFRASTRUCTURE ONLY: drives the reference-side solver adapter
// (cressim-mpm_b200/adapter/gpu_b200_mpm_solver.h) through the reference's own MpmSolverBase /
// MpmSolverGpu interface, in the order SimulationFactoryImpl::createScene and SceneImpl use it
// (src/engine/simulation_factory_impl.cpp:296-349, src/engine/scene_impl.cpp:42-93, 202-220,
// 308-330): stream, particle / material / mask / shape bindings, initialize, computeInitialData,
// step, fetchResults.  Built by `make -C oracle ref-adapter` with the reference's
// src/solver/mpm_solver_gpu.cpp; links libcrmpm_b200.so.
//
//     solver_adapter_check scene.bin steps out.bin
//
// scene.bin (little endian): int32 n, int32 solverType, float32 cell, dt, gmin[3], gmax[3],
// gravity[3], friction, drag, then float32 positionMass[4n], velocity[4n], params0[4n] and int32
// type[n].  The scene has one static ground plane at y = 0.  out.bin: float32 positionMass[4n],
// velocity[4n] after `steps` substeps.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "gpu_b200_mpm_solver.h"

using namespace crmpm;

template <class T> static T *upload(const std::vector<T> &h)
{
    T *d = nullptr;
    cudaMalloc(&d, h.size() * sizeof(T));
    cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

int main(int argc, char **argv)
{
    if (argc < 4)
        return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f)
        return 2;
    int n = 0, type = 0;
    float hdr[13]; // cell, dt, gmin[3], gmax[3], gravity[3], friction, drag
    if (std::fread(&n, 4, 1, f) != 1 || std::fread(&type, 4, 1, f) != 1 || std::fread(hdr, 4, 13, f) != 13)
        return 2;
    std::vector<float4> pm(n), vel(n), mp(n);
    std::vector<int> mt(n);
    if (std::fread(pm.data(), 16, n, f) != (size_t)n || std::fread(vel.data(), 16, n, f) != (size_t)n ||
        std::fread(mp.data(), 16, n, f) != (size_t)n || std::fread(mt.data(), 4, n, f) != (size_t)n)
        return 2;
    std::fclose(f);
    const float cell = hdr[0], dt = hdr[1];
    const int steps = std::atoi(argv[2]);

    // scene-owned particle buffers (SceneImpl) and factory-owned shape / geometry / SDF buffers
    ParticleData pd(n);
    pd.positionMass = upload(pm);
    pd.velocity = reinterpret_cast<Vec3f *>(upload(vel));
    ParticleMaterialData md(n);
    md.params0 = upload(mp);
    md.type = reinterpret_cast<ParticleMaterialType *>(upload(mt));
    unsigned char *mask = upload(std::vector<unsigned char>(n, 1));
    std::vector<unsigned> idx(n);
    for (int i = 0; i < n; ++i)
        idx[i] = (unsigned)i;
    unsigned *dIdx = upload(idx);

    ShapeData sd;
    sd.type = reinterpret_cast<ShapeType *>(upload(std::vector<int>{(int)ShapeType::eStatic}));
    sd.geometryIdx = upload(std::vector<int>{0});
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    sd.position = reinterpret_cast<Vec3f *>(upload(std::vector<float4>{zero}));
    sd.rotation = reinterpret_cast<Quat *>(upload(std::vector<float4>{make_float4(0.f, 0.f, 0.f, 1.f)}));
    sd.invScale = reinterpret_cast<Vec3f *>(upload(std::vector<float4>{make_float4(1.f, 1.f, 1.f, 0.f)}));
    sd.linearVelocity = reinterpret_cast<Vec3f *>(upload(std::vector<float4>{zero}));
    sd.angularVelocity = reinterpret_cast<Vec3f *>(upload(std::vector<float4>{zero}));
    sd.comInvMass = upload(std::vector<float4>{zero});
    sd.inertiaInv0 = upload(std::vector<float4>{zero});
    sd.inertiaInv1 = upload(std::vector<float4>{zero});
    sd.force = upload(std::vector<float4>{zero});
    sd.torque = upload(std::vector<float4>{zero});
    sd.params0 = upload(std::vector<float4>{make_float4(0.f, hdr[12], hdr[11], 0.f)}); // smooth, drag, friction, fatten
    sd.size = 1;
    GeometryData gd;
    gd.type = reinterpret_cast<GeometryType *>(upload(std::vector<int>{(int)GeometryType::ePlane}));
    gd.params0 = upload(std::vector<float4>{zero});
    gd.size = 1;
    GeometrySdfData sdf;
    sdf.dimemsion = reinterpret_cast<Vec3i *>(upload(std::vector<int4>{make_int4(0, 0, 0, 0)}));
    sdf.lowerBoundCellSize = upload(std::vector<float4>{zero});
    sdf.gradientSignedDistance = upload(std::vector<float4>{zero});
    int *ids = upload(std::vector<int>{0});

    Bounds3 bounds(Vec3f(hdr[2], hdr[3], hdr[4]), Vec3f(hdr[5], hdr[6], hdr[7]));
    // created with new and released as the factory does (RefCounted::release deletes it)
    GpuB200MpmSolver *solver = new GpuB200MpmSolver(static_cast<MpmSolverType>(type), n, cell, bounds);
    cudaStream_t stream;
    cudaStreamCreate(&stream);
    solver->setCudaStream(stream);
    solver->bindParticleData(pd);
    solver->bindParticleMaterials(md);
    solver->bindActiveMask(mask);
    solver->setGravity(Vec3f(hdr[8], hdr[9], hdr[10]));
    solver->setIntegrationStepSize(dt);
    solver->setNumActiveParticles((unsigned)n);
    solver->setNumShapes(1);
    solver->bindShapeIds(ids);
    solver->bindShapeData(sd);
    solver->bindGeometryData(gd);
    solver->bindGeometrySdfData(sdf);
    solver->setShapeContactModel(ShapeContactModel::eKinematic);
    solver->initialize();
    solver->computeInitialData((unsigned)n, dIdx);
    for (int s = 0; s < steps; ++s)
        solver->step();
    solver->fetchResults();
    cudaMemcpy(pm.data(), pd.positionMass, 16ull * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(vel.data(), pd.velocity, 16ull * n, cudaMemcpyDeviceToHost);
    solver->release();
    FILE *o = std::fopen(argv[3], "wb");
    if (!o)
        return 2;
    std::fwrite(pm.data(), 16, n, o);
    std::fwrite(vel.data(), 16, n, o);
    std::fclose(o);
    std::printf("steps %d particles %d cuda %s\n", steps, n, cudaGetErrorString(cudaGetLastError()));
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
