"""The C ABI library (CPU-side checks: no compute call needs a GPU here)."""
import os
import re
import subprocess
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "nsx.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nsx_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from nushellx_b200.build import build
    build()
    from nushellx_b200.nsx import load_library
    return load_library()


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert "nsx_matvec" in names and "nsx_solve" in names
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(ROOT, "nushellx_b200", "libnsx.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for n in names:
        assert n in exported, n


def test_python_binding_covers_the_header():
    from nushellx_b200.nsx import SYMBOLS
    assert sorted(SYMBOLS) == declared_functions()


def test_file_code_through_the_abi(lib):
    import ctypes
    buf = ctypes.create_string_buffer(4)
    assert lib.nsx_file_code(2, 3, 33, buf) == 0
    assert buf.value == b"23x"
    assert lib.nsx_file_code(0, 0, 500, buf) != 0


def test_null_arguments_return_errors(lib):
    import ctypes
    h = ctypes.c_void_p()
    assert lib.nsx_create(None, 0, ctypes.byref(h)) < 0
    assert b"null" in lib.nsx_last_error()
    assert lib.nsx_dim(None) == 0
    assert lib.nsx_matvec(None, None, None, 0, None) < 0
    lib.nsx_destroy(None)


def test_missing_files_report_io_error(lib, tmp_path):
    import ctypes
    import numpy as np
    from nushellx_b200.nsx import Files
    f = Files()
    base = str(tmp_path / "nothere").encode()
    f.a = f.b = f.inter = f.like_a = f.like_b = base
    f.xtra = b"x"
    f.nshells, f.nshells_p = 2, 1
    sp = np.ones(2, dtype=np.int32)
    f.shell_parity = sp.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    h = ctypes.c_void_p()
    rc = lib.nsx_load_files(ctypes.byref(f), 0, ctypes.byref(h))
    assert rc == -2
    assert b"cannot open" in lib.nsx_last_error()


def test_fortran_interface_binds_every_entry_point():
    text = open(os.path.join(ROOT, "include", "nsx_iface.f90")).read()
    bound = set(re.findall(r'bind\(C, name="(nsx_[a-z0-9_]+)"\)', text))
    assert bound == set(declared_functions())


def test_ctypes_structs_match_the_c_layout(tmp_path):
    """sizeof/offsetof of every ABI struct from the C compiler equals the Python binding's."""
    import ctypes
    from nushellx_b200 import nsx
    structs = {"nsx_species": nsx.Species, "nsx_problem": nsx.Problem, "nsx_params": nsx.Params,
               "nsx_report": nsx.Report, "nsx_files": nsx.Files, "nsx_stats": nsx.Stats,
               "nsx_dop": nsx.Dop, "nsx_plan_info": nsx.PlanInfo, "nsx_state": nsx.State}
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "nsx.h"', 'int main(void) {']
    for cname, py in structs.items():
        src.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            src.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    src.append("return 0; }")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(out[cname]) == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(out[f"{cname}.{fname}"]) == getattr(py, fname).offset, (cname, fname)
