"""The C-ABI library loads, exports every entry point include/sov_ipm.h declares, and refuses to
compute without an sm_100 device (no CPU fallback). CPU only."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from sovereign_b200 import _lib, abi, problems as P

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "sov_ipm.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sov_[a-z_0-9]+)\s*\(", src)))


def test_header_lists_match():
    assert sorted(_lib.EXPORTS) == declared()


def test_library_exports_every_declared_symbol(lib):
    for name in declared():
        assert hasattr(lib, name), name


def test_struct_layouts_match_header(tmp_path):
    # the sizes and offsets a C compiler gives the header's structs equal the ctypes mirror
    src = tmp_path / "probe.c"
    src.write_text("""#include <stdio.h>
#include <stddef.h>
#include "sov_ipm.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(sov_model), sizeof(sov_options), sizeof(sov_result),
         sizeof(sov_diagnostics), offsetof(sov_result, message), offsetof(sov_options, warm_x),
         offsetof(sov_diagnostics, fp64_fallbacks));
  return 0;
}
""")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [C.sizeof(abi.SovModel), C.sizeof(abi.SovOptions), C.sizeof(abi.SovResult), C.sizeof(abi.SovDiagnostics),
            abi.SovResult.message.offset, abi.SovOptions.warm_x.offset, abi.SovDiagnostics.fp64_fallbacks.offset]
    assert got == want


def test_default_options_match_reference(lib):
    o = abi.SovOptions()
    lib.sov_default_lp_options(C.byref(o))
    assert (o.max_iterations, o.feasibility_tol, o.optimality_tol, o.fraction_to_boundary, o.enable_scaling) == \
        (250, 1e-9, 1e-9, 0.999, 1)
    lib.sov_default_qp_options(C.byref(o))
    assert (o.max_iterations, o.feasibility_tol, o.optimality_tol, o.enable_scaling) == (100, 1e-8, 1e-8, 0)


def test_dims_match_oracle(lib):
    import oracle
    for mdl in (P.bounded_lp_example(), P.reference_staircase(3, 4), P.transport(4, 6, 1)):
        n, m = C.c_int32(), C.c_int32()
        assert lib.sov_ipm_dims(C.byref(mdl.to_abi()), 0, C.byref(n), C.byref(m)) == 0
        f = oracle.ipm_form(mdl)
        assert (n.value, m.value) == (f["n"], f["m"])


def _has_gpu():
    try:
        _lib.device_info()
        return True
    except _lib.SovError:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device behaviour")
def test_no_cpu_fallback_without_device(lib):
    mdl = P.transport(5, 5, 0)
    buf = abi.SovResult()
    rc = lib.sov_lp_solve(C.byref(mdl.to_abi()), None, C.byref(buf))
    assert rc == -2  # SOV_E_NO_DEVICE
    assert buf.status == abi.ERROR and buf.has_objective_value == 0
    x = np.ones(25)
    y = np.zeros(10)
    assert lib.sov_spmv_csc(10, 25, mdl.col_ptr.ctypes.data, mdl.row_idx.ctypes.data, mdl.values.ctypes.data,
                            x.ctypes.data, y.ctypes.data, 0) == -2


def test_bad_arguments_rejected(lib):
    mdl = P.transport(3, 3, 0)
    bad = mdl.to_abi()
    ri = mdl.row_idx.copy()
    ri[0] = 99
    bad.row_idx = abi.iptr(ri)
    buf = abi.SovResult()
    assert lib.sov_lp_solve(C.byref(bad), None, C.byref(buf)) == -1
    assert buf.status == abi.ERROR and b"row index out of range" in buf.message
