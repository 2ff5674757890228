"""The C++ class surface (include/gmg.hpp) driven like the reference's MG checks
(MultiGridPreconditioner::runChecks, include/MultigridPreconditioner.h:311-446)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "grid-mg-bench_b200", "_build", "surface_check")


def test_cpp_surface_runchecks():
    assert os.path.exists(EXE), "build the library first (grid-mg-bench_b200/build.py)"
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all checks passed" in r.stdout
