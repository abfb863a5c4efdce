"""CPU checks of the serving loop: its batch planning and admission rules
(compiled from serve_plan.h into a small test program), and the C ABI's
refusal to start without a GPU."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

import spams_b200
from spams_b200 import _lib

CSRC = os.path.join(ROOT, "spams-devel_b200", "csrc")


def test_plan_and_admission_rules(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path / "serve_plan_test")
    subprocess.run([cxx, "-std=c++17", "-O1", "-I", CSRC,
                    os.path.join(ROOT, "tests", "cpp", "serve_plan_test.cpp"), "-o", exe],
                   check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all checks passed" in r.stdout


def test_server_needs_a_device():
    if spams_b200.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(spams_b200.ScError) as e:
        spams_b200.Server(hbm_budget=1e9)
    assert e.value.status == _lib.SC_ERR_NO_DEVICE


def test_request_records_follow_the_facade_defaults():
    import numpy as np
    X = np.asfortranarray(np.ones((4, 3), np.float32))
    r = spams_b200.request(5, X, "omp", L=3)
    assert (r.dict_id, r.algo, r.n, r.L, r.eps, r.lambda1) == (5, 0, 3, 3, 0.0, 0.0)
    r = spams_b200.request(5, X, "lasso", lambda1=0.2)
    assert (r.algo, r.L, r.mode, r.pos) == (1, -1, 2, 0)
    with pytest.raises(ValueError, match="either provide L, eps or lambda"):
        spams_b200.request(5, X, "omp")
    with pytest.raises(ValueError, match="lambda1 must be defined"):
        spams_b200.request(5, X, "lasso")
    with pytest.raises(ValueError, match="Fortran-ordered float32"):
        spams_b200.request(5, np.ones((4, 3)), "omp", L=2)


def test_minibatch_step_argument_errors_need_no_device():
    with pytest.raises(spams_b200.ScError) as e:
        spams_b200.MinibatchStep(144, 256, 128, mode=7)
    assert e.value.status == _lib.SC_ERR_UNSUPPORTED
    # PENALTY with lambda1 = 0 and a ridge is the reference's conjugate-gradient case
    with pytest.raises(spams_b200.ScError, match="conjugate-gradient"):
        spams_b200.MinibatchStep(144, 256, 128, mode=2, lambda1=0.0, lambda2=0.1)
    with pytest.raises(spams_b200.ScError) as e:
        spams_b200.MinibatchStep(0, 256, 128)
    assert e.value.status == _lib.SC_ERR_INVALID_ARG
