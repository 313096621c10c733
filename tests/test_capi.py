"""The C-ABI boundary: libufvm.so builds, loads and exports every entry point that
include/ufvm.h declares. No compute call is made here (no GPU needed)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "ufvm.h")).read()
    txt = re.sub(r"/\*.*?\*/", " ", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ufvm_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("ufvm_case_create", "ufvm_simple_iteration", "ufvm_compute_residuals_array",
              "ufvm_solve_algebraic_system", "ufvm_agglomerate_level", "ufvm_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol(ufvm_mod):
    lib = ctypes.CDLL(ufvm_mod.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_version_string(ufvm_mod):
    assert b"sm_100a" in ufvm_mod.lib().ufvm_version()


def test_no_cpu_fallback_without_gpu(ufvm_mod):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from matlab_ufvm_b200 import case
    with pytest.raises(ufvm_mod.UfvmError):
        ufvm_mod.GpuCase(case.cavity_case(4))


def test_profile_entry_rejects_bad_arguments(ufvm_mod):
    """The kernel-timing entry point validates its arguments before any device work."""
    lib = ufvm_mod.lib()
    ms, by = ctypes.c_double(), ctypes.c_double()
    P = ctypes.c_void_p
    fake = P(16)  # never dereferenced: every call below is rejected first
    for kernel, n, reps, ptr in ((4, 10, 1, fake), (-1, 10, 1, fake), (0, 0, 1, fake), (0, 10, 0, fake),
                                 (0, 10, 1, P(None))):
        st = lib.ufvm_profile_plain_kernel(kernel, n, ptr, ptr, ptr, ptr, ptr, ptr, reps, ctypes.byref(ms),
                                           ctypes.byref(by), P(None))
        assert st == 1, (kernel, n, reps, st)  # UFVM_E_INVALID
    assert b"bad argument" in lib.ufvm_last_error()
    assert set(ufvm_mod.PLAIN_KERNELS) == {"residual", "SOR", "MCGS", "ILU"}


def _header_struct_fields(name):
    """(field, C type) pairs of a `typedef struct { ... } name;` in include/ufvm.h."""
    txt = open(os.path.join(ROOT, "include", "ufvm.h")).read()
    txt = re.sub(r"/\*.*?\*/", " ", txt, flags=re.S)
    body = re.search(r"typedef struct\s*\{([^}]*)\}\s*" + name + r"\s*;", txt).group(1)
    out = []
    for decl in body.split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        m = re.match(r"((?:const )?[a-z0-9_]+\s*\*?)\s*(.*)", decl)
        ctype, names = m.group(1).replace(" ", ""), m.group(2)
        for nm in names.split(","):
            nm = nm.strip()
            star = nm.startswith("*")
            out.append((nm.lstrip("*").strip(), ctype + ("*" if star else "")))
    return out


@pytest.mark.parametrize("cname,pyname", [("ufvm_mesh_desc", "MeshDesc"), ("ufvm_settings", "Settings")])
def test_ctypes_structs_match_header_layout(ufvm_mod, cname, pyname, tmp_path):
    """The Python mirror's ctypes structs have the header's fields, in order, at the offsets
    the C compiler gives them (a drift here would hand the library shifted settings)."""
    import shutil
    import subprocess
    fields = _header_struct_fields(cname)
    py = getattr(ufvm_mod, pyname)
    assert [f[0] for f in py._fields_] == [f[0] for f in fields]
    for (nm, ctype), (pnm, ptype) in zip(fields, py._fields_):
        if ctype.endswith("*"):
            assert issubclass(ptype, (ctypes._Pointer, ctypes.c_void_p)), nm
        else:
            assert ptype is {"int32_t": ctypes.c_int32, "double": ctypes.c_double}[ctype], nm
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ufvm.h"', "int main(void) {",
             f'  printf("size %zu\\n", sizeof({cname}));']
    lines += [f'  printf("{nm} %zu\\n", offsetof({cname}, {nm}));' for nm, _ in fields]
    lines += ["  return 0;", "}"]
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                       text=True).stdout.splitlines())
    assert int(got["size"]) == ctypes.sizeof(py)
    for nm, _ in fields:
        assert int(got[nm]) == getattr(py, nm).offset, nm


_NULL_CALLS = r'''
import ctypes as ct, sys
sys.path.insert(0, ROOT)
from matlab_ufvm_b200 import ufvm
L = ufvm.lib()
S = ufvm._service_lib()
bad = []
for lib in (L, S):
    for name in NAMES:
        f = getattr(lib, name)
        types = getattr(f, "argtypes", None)
        if not types:
            continue
        args = []
        for t in types:
            if t in (ct.c_int32, ct.c_int, ct.c_int64):
                args.append(0)
            elif t in (ct.c_double, ct.c_float):
                args.append(0.0)
            else:
                args.append(None)
        st = f(*args)
        if st == 0 and name not in OK_ON_NULL:
            bad.append((name, st))
print("BAD", bad)
'''


def test_entry_points_reject_null_handles_and_pointers(ufvm_mod):
    """Every entry point with declared argument types, called with null handles and pointers
    and zero sizes, returns a status instead of dereferencing them (run in a child process, so a
    crash shows as a failure). Only destroy/release of nothing may report success."""
    import subprocess
    import sys
    names = [s for s in declared_symbols() if s not in ("ufvm_version", "ufvm_last_error")]
    ok_on_null = {"ufvm_case_destroy", "ufvm_service_destroy"}
    code = f"ROOT = {ROOT!r}\nNAMES = {names!r}\nOK_ON_NULL = {sorted(ok_on_null)!r}\n" + _NULL_CALLS
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "BAD []" in r.stdout, r.stdout
