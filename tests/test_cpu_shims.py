"""The reference-side bindings compile against the reference's own headers: the cstone primitive shim, the
sph::gpu stage shim and the propagator shim (sphexa_b200/shim/), each with the reference's default SphTypes (float
hydro fields) and with every type FP64. Syntax and template instantiation only (g++ -fsyntax-only); the reference's
single-rank mpi.h stub stands in for MPI, which is absent here. Skipped where the reference sources are absent."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "sphexa_b200", "shim")


def reference_root() -> str:
    return os.environ.get("SPHEXA_REFERENCE", os.path.abspath(os.path.join(ROOT, "..", "reference")))


def cuda_include() -> str:
    for cand in ("/usr/local/cuda/include",):
        if os.path.exists(os.path.join(cand, "cuda_runtime.h")):
            return cand
    pytest.skip("cuda_runtime.h not found")


def compile_syntax(src: str, stub_dir: str):
    ref = reference_root()
    if not os.path.isdir(os.path.join(ref, "sph", "include")):
        pytest.skip("reference sources not present")
    if shutil.which("g++") is None:
        pytest.skip("g++ not found")
    cmd = ["g++", "-std=c++20", "-fsyntax-only", "-fopenmp", "-include", "map", "-include", "sstream",
           "-I" + os.path.join(ROOT, "include"), "-I" + SHIM, "-I" + stub_dir,
           "-I" + os.path.join(ref, "domain", "include"), "-I" + os.path.join(ref, "sph", "include"),
           "-I" + os.path.join(ref, "main", "src"), "-I" + os.path.join(ref, "physics", "cooling", "include"),
           "-I" + ref, "-I" + cuda_include(), src]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-4000:]


@pytest.fixture(params=["reference_types", "fp64_types"])
def stub_dir(request, tmp_path):
    """the single-rank mpi.h stub alone (the reference's own sph/types.hpp), or with the FP64 types override"""
    stub = os.path.join(ROOT, "oracle", "ref", "stub")
    if request.param == "fp64_types":
        return stub
    d = tmp_path / "stub"
    d.mkdir()
    shutil.copy(os.path.join(stub, "mpi.h"), d / "mpi.h")
    return str(d)


def test_cstone_primitive_shim_compiles(stub_dir):
    compile_syntax(os.path.join(SHIM, "cstone_gpu_sphb.cpp"), stub_dir)


def test_sph_gpu_stage_shim_compiles(stub_dir):
    compile_syntax(os.path.join(SHIM, "sph_gpu_sphb.cpp"), stub_dir)


def test_propagator_shim_compiles(stub_dir, tmp_path):
    tu = tmp_path / "propagator_tu.cpp"
    tu.write_text('#include "cstone/domain/domain.hpp"\n'
                  '#include "sphexa/simulation_data.hpp"\n'
                  '#include "ve_hydro_sphb.hpp"\n'
                  "template class sphexa::HydroVeSphbProp<false, cstone::Domain<uint64_t, double, cstone::CpuTag>,\n"
                  "                                       sphexa::SimulationData<cstone::CpuTag>>;\n"
                  "template class sphexa::HydroVeSphbProp<true, cstone::Domain<uint64_t, double, cstone::CpuTag>,\n"
                  "                                       sphexa::SimulationData<cstone::CpuTag>>;\n")
    compile_syntax(str(tu), stub_dir)
