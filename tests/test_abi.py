"""The C-ABI library loads and exports every symbol include/wnlqg_b200.h declares (no compute)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def header_functions():
    text = open(os.path.join(ROOT, "include", "wnlqg_b200.h")).read()
    return sorted(set(re.findall(r"\b(wnlqg_b200_[a-z_]+)\s*\(", text)))


def test_header_and_loader_agree():
    from wanniernlqg_b200 import _lib
    assert sorted(_lib.EXPORTED_SYMBOLS) == header_functions()


def test_library_exports_all_symbols():
    from wanniernlqg_b200 import build, _lib
    build.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for name in header_functions():
        assert hasattr(lib, name), name
    L = _lib.load()
    assert L.wnlqg_b200_version().startswith(b"wnlqg-b200")


def test_struct_sizes_match_c():
    """ctypes layouts equal the C layouts (compiled with the same header)."""
    import subprocess
    import tempfile
    from wanniernlqg_b200 import _abi
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "wnlqg_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(wnlqg_model_desc), sizeof(wnlqg_response_request),
         sizeof(wnlqg_task_desc), offsetof(wnlqg_task_desc, fermi_energy), offsetof(wnlqg_task_desc, precision),
         offsetof(wnlqg_task_desc, fermi_surface_broadening), offsetof(wnlqg_task_desc, wannier_center_convention),
         sizeof(wnlqg_autotune_report), offsetof(wnlqg_autotune_report, response_ms),
         offsetof(wnlqg_autotune_report, warm_start), offsetof(wnlqg_autotune_report, start_ms),
         offsetof(wnlqg_autotune_report, width_ms), offsetof(wnlqg_autotune_report, shg_grid_ms),
         offsetof(wnlqg_autotune_report, eigh_grid_ms), offsetof(wnlqg_task_desc, spectral_gap_tolerance),
         offsetof(wnlqg_task_desc, linear_transport_gamma_inter), offsetof(wnlqg_task_desc, finite_difference_step),
         offsetof(wnlqg_task_desc, derivative_backend));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    got = [ctypes.sizeof(_abi.ModelDesc), ctypes.sizeof(_abi.ResponseRequest), ctypes.sizeof(_abi.TaskDesc),
           _abi.TaskDesc.fermi_energy.offset, _abi.TaskDesc.precision.offset,
           _abi.TaskDesc.fermi_surface_broadening.offset, _abi.TaskDesc.wannier_center_convention.offset,
           ctypes.sizeof(_abi.AutotuneReport), _abi.AutotuneReport.response_ms.offset,
           _abi.AutotuneReport.warm_start.offset, _abi.AutotuneReport.start_ms.offset,
           _abi.AutotuneReport.width_ms.offset, _abi.AutotuneReport.shg_grid_ms.offset,
           _abi.AutotuneReport.eigh_grid_ms.offset, _abi.TaskDesc.spectral_gap_tolerance.offset,
           _abi.TaskDesc.linear_transport_gamma_inter.offset, _abi.TaskDesc.finite_difference_step.offset,
           _abi.TaskDesc.derivative_backend.offset]
    assert [int(x) for x in out] == got
