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
