"""The split search's work-item planner, host logic only: tests/cpp/plan_items.cu is compiled with nvcc
(host code; the planner's header pulls in device declarations) against the in-tree library and run on
the CPU. It covers the sample-chunk groups of the top levels and their memory limit."""
import os
import shutil
import subprocess

import pytest

from curfil_b200 import _build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_plan_level_items_invariants(tmp_path):
    if not os.path.exists(_build.NVCC) and shutil.which("nvcc") is None:
        pytest.skip("nvcc not available")
    lib = _build.build()
    libdir = os.path.dirname(lib)
    exe = str(tmp_path / "plan_items")
    cmd = [_build.NVCC] + _build.ARCH + ["-std=c++17", "-O1", "--expt-relaxed-constexpr", "-I",
                                         os.path.join(ROOT, "include"),
                                         os.path.join(ROOT, "tests", "cpp", "plan_items.cu"), "-L", libdir,
                                         "-lcurfil_b200", "-Xlinker", "-rpath", "-Xlinker", libdir, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    run = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "0 failures" in run.stdout
