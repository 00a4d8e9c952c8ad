"""The reference-side adapter (include/sov_ipm_adapter.hpp).

* CPU: it compiles against the reference's own types.hpp and links with libsovipm.so and the
  reference core; on a machine without an sm_100 GPU the call comes back as SolverStatus::Error
  naming the device, never as a CPU answer (needs the reference headers).
* GPU: oracle/_ref/adapter_check (tests/adapter_check.cpp, built with the reference library by
  oracle/Makefile) runs solve_lp, solve_qp, solve_lp_batch and solve_branch_children on name-keyed
  OptimizationModels next to the reference's InteriorPointSolver / QpInteriorPointSolver and
  compares status, objective, the primal and dual maps and lp_diagnostics["ipm"]."""
import os
import subprocess

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(oracle.REFERENCE_DIR, "solver")

ADAPTER_CHECK = os.path.join(ROOT, "oracle", "_ref", "adapter_check")
needs_headers = pytest.mark.skipif(not os.path.isdir(REF), reason="reference headers not present")

PROGRAM = r"""
#include <cstdio>
#include "sov_ipm_adapter.hpp"
using namespace sovereign;
int main() {
  OptimizationModel m;
  m.problem_type = ProblemType::LP;
  m.sense = Sense::Minimize;
  for (const char* v : {"a", "b"}) { Variable x; x.name = v; m.variables.push_back(x); }
  m.objective.linear = {{"a", 1.0}, {"b", 2.0}};
  Constraint c; c.name = "c"; c.linear = {{"a", 1.0}, {"b", 1.0}}; c.sense = ConstraintSense::Ge; c.rhs = 1.0;
  m.constraints.push_back(c);
  SolverResult r = b200::solve_lp(m);
  Constraint bad; bad.linear = {{"zz", 1.0}};
  m.constraints.push_back(bad);
  SolverResult e = b200::solve_lp(m);
  std::printf("%d|%s|%d|%s\n", static_cast<int>(r.status), r.message.c_str(), static_cast<int>(e.status),
              e.message.c_str());
  return 0;
}
"""


@needs_headers
def test_adapter_compiles_links_and_reports_errors(tmp_path):
    from sovereign_b200 import _lib
    _lib.load()
    src = tmp_path / "adapter_probe.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "adapter_probe"
    lib_dir = os.path.join(ROOT, "sovereign_b200")
    cmd = ["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(REF, "core/include"),
           str(src), os.path.join(REF, "core/src/types.cpp"), "-L" + lib_dir, "-lsovipm",
           "-Wl,-rpath," + lib_dir, "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.strip().split("|")
    status, msg, bad_status, bad_msg = int(out[0]), out[1], int(out[2]), out[3]
    assert bad_status == 7 and bad_msg == "IPM error: Unknown variable in constraint: zz"
    has_gpu = True
    try:
        _lib.device_info()
    except _lib.SovError:
        has_gpu = False
    if has_gpu:
        assert status == 0  # OPTIMAL
    else:
        assert status == 7 and "no CUDA device" in msg


@pytest.mark.skipif(not os.path.exists(ADAPTER_CHECK), reason="adapter check not built (needs the reference)")
def test_adapter_check_models_solve_in_the_reference():
    r = subprocess.run([ADAPTER_CHECK, "--reference-only"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "failures 0" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_adapter_matches_reference_solvers_on_gpu():
    assert os.path.exists(ADAPTER_CHECK), "oracle/_ref/adapter_check is built with the reference library"
    r = subprocess.run([ADAPTER_CHECK], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "failures 0" in r.stdout, r.stdout + r.stderr
