"""The C++ half of the drop-in boundary: the qkrylov reference's own C++
test programs (tests/*.cpp of the reference, listed in its
tests/CMakeLists.txt:1-26), compiled unchanged against this library's
headers and linked to libqkrylov_b200.so by tests/ref_cxx/Makefile, must
each exit 0 on the GPU.  They assert with NDEBUG undefined, so an exit code
of 0 means every assertion of the reference's test held.  Skipped where the
executables were not built (no reference checkout on the build machine)."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "ref_cxx", "_bin")
TESTS = ["test_hamiltonian_sz", "test_heisenberg_2site", "test_lanczos_2site", "test_opsum", "test_spinhalf_basis",
         "test_spinhalf_site", "test_vector_ops", "test_fermion_basis", "test_fermion_site", "test_davidson",
         "test_lanczos_ritz", "test_dynamics", "test_tj_basis", "test_tj_site", "test_ftlm", "test_workflow",
         "test_c_api"]

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.isdir(BIN), reason="reference C++ tests not built (tests/ref_cxx)")]


@pytest.mark.parametrize("name", TESTS)
def test_reference_cxx_program_passes(name):
    exe = os.path.join(BIN, name)
    assert os.path.exists(exe), f"{name} was not built"
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, f"{name} exited {r.returncode}\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}"
