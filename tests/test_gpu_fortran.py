"""The Fortran front end (cosmokdtree_b200/fortran) compiled against libckd.so and
run against brute force, when a Fortran compiler is available (none is installed
in the build image; the test is skipped there)."""
import os
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FDIR = os.path.join(HERE, "..", "cosmokdtree_b200", "fortran")


def _compiler():
    for c in ("gfortran", "flang-new", "flang", "ifx", "nvfortran"):
        if shutil.which(c):
            return c
    return None


def test_gpu_fortran_front_end(gpu, tmp_path):
    fc = _compiler()
    if fc is None:
        pytest.skip("no Fortran compiler on this machine")
    lib = os.path.dirname(gpu._lib.LIB_PATH)
    exe = str(tmp_path / "test_front_end")
    flags = ["-O2", "-ffp-contract=off"] if fc == "gfortran" else ["-O2"]
    subprocess.run([fc, *flags, "-J", str(tmp_path), os.path.join(FDIR, "cosmokdtree_gpu.f90"),
                    os.path.join(FDIR, "test_cosmokdtree_gpu.f90"), "-L" + lib, "-lckd",
                    "-Wl,-rpath," + lib, "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True)
    assert "OK" in out.stdout
