"""The C ABI without a GPU: every entry point declared in include/swm.h is
exported by libswm.so, the ctypes structs match the C layout, argument
validation answers before any CUDA call, and the Fortran interface module
binds every entry point by its C name."""
import ctypes
import os
import re
import subprocess

import pytest

import swm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "swm.h")
F90 = os.path.join(ROOT, "sw-mpdec_b200", "fortran", "mod_swm_capi.f90")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"SWM_API\s+[\w\s\*]*?\b(swm_\w+)\s*\(", src)))


def test_header_declarations_match_binding():
    assert declared() == sorted(swm.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(swm.LIB_PATH)
    for name in declared():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", swm.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (swm_\w+)", out))
    assert set(declared()) <= exported


def c_layout(struct, fields, d):
    prog = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(){",
            f'printf("%zu\\n", sizeof({struct}));']
    prog += [f'printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    prog += ["return 0;}"]
    src, exe = os.path.join(d, f"{struct}.c"), os.path.join(d, f"{struct}.bin")
    open(src, "w").write("\n".join(prog))
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, src, "-o", exe], check=True)
    vals = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    return vals[0], vals[1:]


@pytest.mark.parametrize("struct,cls", [("swm_params", swm.SwmParams),
                                        ("swm_stats", swm.SwmStats)])
def test_struct_layout_matches_ctypes(struct, cls, tmp_path):
    names = [f[0] for f in cls._fields_]
    size, offs = c_layout(struct, names, str(tmp_path))
    assert size == ctypes.sizeof(cls)
    assert offs == [getattr(cls, n).offset for n in names]


def test_params_default_and_validation_without_gpu():
    lib = swm.load()
    p = swm.make_params(64, 32, (0.0, 0.0), (2.0, 1.0))
    assert (p.cfl, p.timescheme, p.jacobi_maxiter, p.jacobi_tol) == (1.0, 5, 1000, 1e-16)
    h = ctypes.c_void_p()
    bad = swm.make_params(2, 32, (0.0, 0.0), (2.0, 1.0))
    assert lib.swm_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    bad = swm.make_params(64, 32, (0.0, 0.0), (2.0, 1.0), timescheme=8)
    assert lib.swm_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    assert b"timescheme" in lib.swm_last_error()
    bad = swm.make_params(64, 32, (0.0, 0.0), (2.0, 1.0), jacobi_block=9)
    assert lib.swm_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    assert lib.swm_strerror(1) == b"Jacobi not converged (maxIter reached)"
    assert lib.swm_destroy(None) == 0


def test_null_handle_calls_fail_cleanly():
    lib = swm.load()
    dt = ctypes.c_double()
    assert lib.swm_timestep(None, ctypes.byref(dt)) == -1
    assert lib.swm_step(None, 0.0, 1e-3) == -1
    assert lib.swm_set_state(None, None) == -1


def test_fortran_module_binds_every_entry_point():
    src = open(F90).read().lower()
    bound = set(re.findall(r'bind\s*\(\s*c\s*,\s*name\s*=\s*"(swm_\w+)"', src))
    core = {"swm_params_default", "swm_create", "swm_destroy", "swm_set_state", "swm_get_state",
            "swm_set_wb_state", "swm_timestep", "swm_step", "swm_get_stats", "swm_last_error"}
    assert core <= bound
    assert bound <= set(declared())


def test_normal_build_has_no_checked_records():
    # the index checks exist only in libswm_checked.so; the product library says so
    # without touching a GPU
    with pytest.raises(swm.SwmError) as e:
        swm.checked_status()
    assert e.value.code == -7
