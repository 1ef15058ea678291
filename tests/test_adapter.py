"""The reference-side drop-in adapter compiles against the reference's own solver headers.

cressim-mpm_b200/adapter/gpu_b200_mpm_solver.h derives from the reference's MpmSolverGpu and checks
at compile time that the C-ABI descriptors have the reference's struct layouts.  Needs the
reference sources (skipped where they are absent).
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
import oracle_py  # noqa: E402

# the reference's sources, where the oracle recipe (oracle/Makefile print-ref) finds them
REF = oracle_py.reference_root() or ""


@pytest.mark.skipif(not REF, reason="reference sources not present (oracle/Makefile print-ref)")
def test_adapter_compiles_against_reference_headers(tmp_path):
    src = tmp_path / "use_adapter.cpp"
    src.write_text('#include "gpu_b200_mpm_solver.h"\n'
                   "crmpm::MpmSolverGpu *make(crmpm::Bounds3 b) {\n"
                   "  return new crmpm::GpuB200MpmSolver(crmpm::MpmSolverType::eGpuMlsMpmSolver, 1000, 0.05f, b);\n}\n")
    inc = ["include/math", "include/utils", "include/core", "include/solver", "include/engine",
           "include/geometry_utils", "src/solver", "src/core", "src/utils"]
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-w", f"-I{ROOT}/include", f"-I{ROOT}/cressim-mpm_b200/adapter"]
    cmd += [f"-I{REF}/{d}" for d in inc] + [str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


@pytest.mark.skipif(not REF, reason="reference sources not present (oracle/Makefile print-ref)")
def test_sdf_adapter_compiles_against_reference_headers(tmp_path):
    """cressim-mpm_b200/adapter/gpu_b200_sdf_builder.h: the GPU SDF build behind the reference's
    SdfBuilder calls, with SdfDesc / TriangleMesh converted field by field."""
    src = tmp_path / "use_sdf_adapter.cpp"
    src.write_text('#include "gpu_b200_sdf_builder.h"\n'
                   "void build(crmpm::SdfDesc &d, crmpm::TriangleMesh &m, float4 *out, float4 *outMod) {\n"
                   "  crmpm::GpuB200SdfBuilder::precomputeSdfDesc(d, m);\n"
                   "  crmpm::GpuB200SdfBuilder::computeSdfWithGradient(d, m, out);\n"
                   "  crmpm::GpuB200SdfBuilder::computeModSdfWithGradient(d, m, outMod);\n}\n")
    inc = ["include/math", "include/utils", "include/core", "include/solver", "include/engine",
           "include/geometry_utils", "src/solver", "src/core", "src/utils"]
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-w", f"-I{ROOT}/include", f"-I{ROOT}/cressim-mpm_b200/adapter",
           "-I/usr/local/cuda/include"]
    cmd += [f"-I{REF}/{d}" for d in inc] + [str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


ADAPTER_HOST_PROGRAM = r'''
// Drives GpuB200MlsMpmSolver through the reference's MpmSolverBase members against a counting stub
// of the C ABI (no GPU): initialize sends every setting once; a step afterwards calls only
// CrB200SolverStep unless a setting changed; a shape array the factory regrew in place is sent again.
#include <cstdio>
#include "gpu_b200_mpm_solver.h"

enum { C_STEP, C_GRAV, C_DT, C_ITER, C_CM, C_NACT, C_NSH, C_IDS, C_SD, C_GD, C_SDF, C_OTHER, C_N };
static int calls[C_N];
static void *lastPosition = nullptr;
#define H CrB200SolverHandle
extern "C" {
const char *CrB200GetLastError(void) { return ""; }
int CrB200SolverCreate(int, int, float, const float *, const float *, void *, H *out)
{ ++calls[C_OTHER]; *out = reinterpret_cast<H>(0x10); return 0; }
int CrB200SolverRelease(H) { return 0; }
int CrB200SolverInitialize(H) { ++calls[C_OTHER]; return 0; }
int CrB200SolverStep(H, float *) { ++calls[C_STEP]; return 0; }
int CrB200SolverComputeInitialData(H, unsigned int, const unsigned int *) { return 0; }
int CrB200SolverSetGravity(H, float, float, float) { ++calls[C_GRAV]; return 0; }
int CrB200SolverSetIntegrationStepSize(H, float) { ++calls[C_DT]; return 0; }
int CrB200SolverSetSolverIterations(H, int) { ++calls[C_ITER]; return 0; }
int CrB200SolverSetShapeContactModel(H, int) { ++calls[C_CM]; return 0; }
int CrB200SolverSetNumActiveParticles(H, unsigned int) { ++calls[C_NACT]; return 0; }
int CrB200SolverBindParticleData(H, CrB200Float4 *, CrB200Float4 *) { ++calls[C_OTHER]; return 0; }
int CrB200SolverBindParticleMaterials(H, CrB200Float4 *, int *) { ++calls[C_OTHER]; return 0; }
int CrB200SolverBindActiveMask(H, unsigned char *) { ++calls[C_OTHER]; return 0; }
int CrB200SolverSetNumShapes(H, int) { ++calls[C_NSH]; return 0; }
int CrB200SolverBindShapeIds(H, int *) { ++calls[C_IDS]; return 0; }
int CrB200SolverBindShapeData(H, const CrB200ShapeData *s)
{ ++calls[C_SD]; lastPosition = (void *)s->position; return 0; }
int CrB200SolverBindGeometryData(H, const CrB200GeometryData *) { ++calls[C_GD]; return 0; }
int CrB200SolverBindGeometrySdfData(H, const CrB200GeometrySdfData *) { ++calls[C_SDF]; return 0; }
int CrB200SolverSetOption(H, int, int) { ++calls[C_OTHER]; return 0; }
}

static int total() { int t = 0; for (int k = 0; k < C_N; ++k) t += calls[k]; return t; }
static void reset() { for (int k = 0; k < C_N; ++k) calls[k] = 0; }
#define EXPECT(c) do { if (!(c)) { std::printf("FAILED %s (line %d)\n", #c, __LINE__); return 1; } } while (0)

int main()
{
    using namespace crmpm;
    GpuB200MlsMpmSolver s(1000, 0.01f, Bounds3(Vec3f(-1, -1, -1), Vec3f(1, 1, 1)));
    ParticleData pd(1000);
    pd.positionMass = reinterpret_cast<float4 *>(0x1000);
    pd.velocity = reinterpret_cast<Vec3f *>(0x2000);
    ParticleMaterialData md(1000);
    md.params0 = reinterpret_cast<float4 *>(0x3000);
    md.type = reinterpret_cast<ParticleMaterialType *>(0x4000);
    unsigned char *mask = reinterpret_cast<unsigned char *>(0x5000);
    int *ids = reinterpret_cast<int *>(0x6000);
    ShapeData sd{};
    sd.position = reinterpret_cast<Vec3f *>(0x7000);
    GeometryData gd{};
    GeometrySdfData sdf{};
    s.bindParticleData(pd);
    s.bindParticleMaterials(md);
    s.bindActiveMask(mask);
    s.setNumActiveParticles(1000);
    s.setNumShapes(2);
    s.bindShapeIds(ids);
    s.bindShapeData(sd);
    s.bindGeometryData(gd);
    s.bindGeometrySdfData(sdf);
    s.setGravity(Vec3f(0, -9.81f, 0));
    s.setIntegrationStepSize(1e-4f);
    s.initialize();
    EXPECT(calls[C_GRAV] == 1 && calls[C_DT] == 1 && calls[C_NACT] == 1 && calls[C_SD] == 1 && calls[C_SDF] == 1);
    reset();
    for (int k = 0; k < 10; ++k)
        s.step();
    EXPECT(calls[C_STEP] == 10 && total() == 10);        // nothing changed: one C-ABI call a substep
    EXPECT(s.abiCalls() > 10);                            // the set-up calls are counted too
    reset();
    s.setGravity(Vec3f(0, -9.0f, 0));
    s.setNumActiveParticles(900);
    s.step();
    EXPECT(calls[C_GRAV] == 1 && calls[C_NACT] == 1 && calls[C_STEP] == 1 && total() == 3);
    reset();
    sd.position = reinterpret_cast<Vec3f *>(0x8000);      // the factory regrew its shape arrays
    s.step();
    EXPECT(calls[C_SD] == 1 && lastPosition == (void *)0x8000 && total() == 2);
    reset();
    s.setNumShapes(0);
    s.step();
    EXPECT(calls[C_NSH] == 1 && calls[C_SD] == 0 && total() == 2);
    std::printf("OK\n");
    return 0;
}
'''


@pytest.mark.skipif(not REF, reason="reference sources not present (oracle/Makefile print-ref)")
def test_adapter_sends_only_changed_settings(tmp_path):
    """The drop-in adapter's host cost per substep: after initialize, a step crosses the C ABI once
    unless a setting changed, and a shape descriptor whose arrays were regrown is sent again
    (a counting stub of the C ABI stands in for the engine; no GPU)."""
    src = tmp_path / "adapter_host.cpp"
    src.write_text(ADAPTER_HOST_PROGRAM)
    exe = tmp_path / "adapter_host"
    inc = ["include/math", "include/utils", "include/core", "include/solver", "include/engine",
           "include/geometry_utils", "src/solver", "src/core", "src/utils"]
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cmd = ["g++", "-std=c++17", "-O1", "-w", f"-I{ROOT}/include", f"-I{ROOT}/cressim-mpm_b200/adapter",
           f"-I{cuda}/include"]
    cmd += [f"-I{REF}/{d}" for d in inc]
    cmd += [str(src), f"{REF}/src/solver/mpm_solver_gpu.cpp", "-o", str(exe), f"-L{cuda}/lib64", "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout + r.stderr
