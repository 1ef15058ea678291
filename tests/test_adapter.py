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
