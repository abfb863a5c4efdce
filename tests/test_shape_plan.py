"""CPU checks of the coding kernels' launch-shape planning and the autotuner's
choice rule (shape_plan.h, compiled with the engine's state-size functions
into a small test program)."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

CSRC = os.path.join(ROOT, "spams-devel_b200", "csrc")
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")


def test_launch_shapes_and_tuner_rule(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    if not os.path.exists(os.path.join(CUDA_INC, "cuda_runtime.h")):
        pytest.skip("CUDA headers not found")
    exe = str(tmp_path / "shape_plan_test")
    subprocess.run([cxx, "-std=c++17", "-O1", "-I", CSRC, "-I", os.path.join(ROOT, "include"),
                    "-I", CUDA_INC, os.path.join(ROOT, "tests", "cpp", "shape_plan_test.cpp"),
                    "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all checks passed" in r.stdout
