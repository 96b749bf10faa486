"""The C++ interface (include/curfil_b200.hpp), the reference's classes over the C-ABI.

tests/cpp/test_api.cpp is compiled with g++ against the in-tree library and run in groups: the host
behaviour here on the CPU, the known-answer and end-to-end tests (train, predict, export/import
against the C-ABI's own forest) on the GPU. The C++ Sampler is checked draw for draw against the
oracle's restatement of the reference's Sampler.
"""
import os
import subprocess

import numpy as np
import pytest

from curfil_b200 import _build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def test_binary(tmp_path_factory):
    lib = _build.build()
    out = str(tmp_path_factory.mktemp("cpp") / "test_api")
    libdir = os.path.dirname(lib)
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "test_api.cpp"), "-L", libdir, "-lcurfil_b200",
           "-Wl,-rpath," + libdir, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return out


def run(binary, *args, timeout=600):
    r = subprocess.run([binary] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout)
    return r.returncode, r.stdout, r.stderr


def test_cpp_host_behaviour(test_binary):
    rc, out, err = run(test_binary, "--group", "cpu")
    assert rc == 0, out + err
    assert "0 failures" in out


def test_cpp_gpu_work_fails_loudly_without_a_gpu(test_binary):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    rc, out, err = run(test_binary, "--group", "nogpu")
    assert rc == 0, out + err


@pytest.mark.parametrize("seed,lo,hi", [(7, 0, 99), (4711, 0, 0xFFFF - 1), (123, 0, 0xFFFFFF - 1), (5, -3, 3)])
def test_cpp_sampler_matches_oracle(test_binary, seed, lo, hi):
    from oracle import pyoracle as orc
    rc, out, err = run(test_binary, "--sampler", seed, lo, hi, 200)
    assert rc == 0, err
    got = np.array([int(v) for v in out.split()], np.int64)
    np.testing.assert_array_equal(got, np.asarray(orc.sampler_draws(seed, lo, hi, 200), np.int64))


@pytest.mark.gpu
def test_cpp_known_answers_and_end_to_end(test_binary):
    rc, out, err = run(test_binary, "--group", "gpu", timeout=1200)
    assert rc == 0, out + err
    assert "0 failures" in out
