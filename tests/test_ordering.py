"""Host ordering, symbolic analysis and GPU work schedule of the sparse L D L', compiled with g++ from
sovereign_b200/csrc/sparse.cpp (no GPU): the approximate minimum-degree order is a permutation,
the patterns of L equal a brute-force symbolic elimination in that order, the elimination tree and
the level schedule are consistent, and the 130 x 130 grid's fill stays near the reference's."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_ordering_and_symbolic_analysis(tmp_path):
    exe = tmp_path / "ordering_check"
    csrc = os.path.join(ROOT, "sovereign_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I" + csrc,
                    os.path.join(ROOT, "tests", "ordering_check.cpp"), os.path.join(csrc, "sparse.cpp"),
                    os.path.join(csrc, "stdform.cpp"), "-o", str(exe), "-lpthread"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "failures 0" in r.stdout


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_gpu_work_schedule_walked_on_the_host(tmp_path):
    # sparse_schedule's pieces and combine steps, walked on the CPU as the GPU kernels walk them:
    # every term covered once, and the factor and solves reproduce K x = b to 1e-13 (backward error)
    exe = tmp_path / "schedule_check"
    csrc = os.path.join(ROOT, "sovereign_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I" + csrc,
                    os.path.join(ROOT, "tests", "schedule_check.cpp"), os.path.join(csrc, "sparse.cpp"),
                    "-o", str(exe), "-lpthread"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "failures 0" in r.stdout
