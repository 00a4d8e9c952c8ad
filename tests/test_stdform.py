"""Host standard form and gather map, compiled with g++ from sovereign_b200/csrc/stdform.cpp (no GPU):
the batched path's in-place builder must equal the general one bit for bit, and the dense gather
map must give every target the generic builder's contributions in the same order."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_in_place_standard_form_is_bit_identical(tmp_path):
    exe = tmp_path / "stdform_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
                    "-I" + os.path.join(ROOT, "sovereign_b200", "csrc"), os.path.join(ROOT, "tests", "stdform_check.cpp"),
                    os.path.join(ROOT, "sovereign_b200", "csrc", "stdform.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches 0" in r.stdout


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_dense_gather_map_matches_generic_builder(tmp_path):
    exe = tmp_path / "assembly_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
                    "-I" + os.path.join(ROOT, "sovereign_b200", "csrc"), os.path.join(ROOT, "tests", "assembly_check.cpp"),
                    os.path.join(ROOT, "sovereign_b200", "csrc", "stdform.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches 0" in r.stdout
