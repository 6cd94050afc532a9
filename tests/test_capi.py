"""The C-ABI library loads and exports every entry point include/*.h
declares; host-side argument checks fail loudly without touching a GPU."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(mhd_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared_symbols()
    assert "mhd_step" in names and "mhd_ctx_create" in names and len(names) >= 15


@pytest.mark.parametrize("name", declared_symbols())
def test_library_exports(name):
    from mpcns_mercury_b200 import capi

    L = capi.lib()
    assert hasattr(L, name), name


def test_bad_arguments_return_status():
    from mpcns_mercury_b200 import capi

    L = capi.lib()
    out = ctypes.c_void_p()
    assert L.mhd_ctx_create(None, ctypes.byref(out)) == 1  # MHD_ERR_ARG
    assert b"bad descriptor" in L.mhd_last_error()
    nc, loc = ctypes.c_int32(), ctypes.c_int32()
    assert L.mhd_field_info(999, ctypes.byref(nc), ctypes.byref(loc)) == 1
    assert L.mhd_field_info(capi.FIELD_ID["JCELL_W"], ctypes.byref(nc), ctypes.byref(loc)) == 0
    assert nc.value == 36 and loc.value == 0
    t = ctypes.c_void_p()
    assert L.mhd_topology_periodic_block(capi._i3([1, 4, 4]), 4, ctypes.byref(t)) == 1


def test_struct_layouts_match_header(tmp_path):
    """ctypes mirrors of the header structs have the C sizes."""
    import subprocess

    from mpcns_mercury_b200 import capi

    src = ('#include <stdio.h>\n#include "mercury_mhd.h"\nint main(){printf("%zu %zu %zu %zu %zu %zu %zu",'
           'sizeof(mhd_desc),sizeof(mhd_constants),sizeof(mhd_copy),sizeof(mhd_info),sizeof(mhd_alias_classes),'
           'sizeof(mhd_restart_image),sizeof(mhd_tecplot_image));}')
    c = str(tmp_path / "s.c")
    open(c, "w").write(src)
    exe = str(tmp_path / "s")
    subprocess.check_call(["gcc", "-I" + os.path.join(ROOT, "include"), c, "-o", exe])
    got = [int(x) for x in subprocess.check_output([exe]).split()]
    want = [ctypes.sizeof(capi.MhdDesc), ctypes.sizeof(capi.MhdConstants), ctypes.sizeof(capi.MhdCopy),
            ctypes.sizeof(capi.MhdInfo), ctypes.sizeof(capi.MhdAliasClasses), ctypes.sizeof(capi.MhdRestartImage),
            ctypes.sizeof(capi.MhdTecplotImage)]
    assert got == want


def test_mixed_resistive_solve_counts_its_fp64_companion():
    """mhd_desc_device_bytes of a mixed-precision solve with the implicit
    substep includes the FP64 companion that holds the refinement's residual."""
    from mpcns_mercury_b200 import reference_constants
    from mpcns_mercury_b200.capi import SolveDesc

    cells = [(16, 16, 16)]
    res, plain = reference_constants(cfl=0.4, resistive=True), reference_constants(cfl=0.4)
    by = {}
    for key, k, prec in (("mixed_res", res, 1), ("mixed", plain, 1), ("fp64_res", res, 0), ("fp64", plain, 0)):
        d = SolveDesc(cells, 3, k, precision=prec)
        by[key] = d.device_bytes()
        d.close()
    # the substep's 18 work arrays: 8 bytes each in FP64, 4 in mixed
    res_arrays_fp64 = by["fp64_res"] - by["fp64"]
    assert res_arrays_fp64 > 0
    assert by["mixed_res"] == by["mixed"] + res_arrays_fp64 // 2 + by["fp64_res"]
