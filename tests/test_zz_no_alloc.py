"""ufvm_solve_sor_noalloc (the smoother with its scratch in a fixed array inside the library)
against ufvm_solve_sor, through the C-ABI: two calls in a row on systems of different sizes,
each compared bit for bit with the allocating entry point, plus the size limit. Collected last
so that it also runs after the other GPU tests in the same process."""
import ctypes as ct

import numpy as np
import pytest

from helpers import random_diag_dominant

MAX_ROWS = 262144


def _dev(torch, a, dt):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).cuda()


def _system(torch, rowptr, col, ac, anb, bc, x0):
    return [_dev(torch, rowptr, np.int32), _dev(torch, col, np.int32), _dev(torch, ac, np.float64),
            _dev(torch, anb, np.float64), _dev(torch, bc, np.float64), _dev(torch, x0, np.float64)]


def _call(lib, fn, n, arrs, stream):
    ptrs = [ct.c_void_p(t.data_ptr()) for t in arrs]
    return getattr(lib, fn)(n, *ptrs, ct.c_void_p(stream))


@pytest.mark.gpu
def test_noalloc_sor_matches_allocating_sor_twice(ufvm_mod, oracle_mod):
    import torch
    from matlab_ufvm_b200 import case
    lib = ufvm_mod.lib()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(7)
    # first call: a larger random system; second call: the smaller pressure-correction system
    # of a 48 x 48 cavity, so the second call runs on scratch that still holds the first
    # call's schedule
    systems = [random_diag_dominant(20000, 3, nbr=6)]
    oc = oracle_mod.OracleCase(case.cavity_case(48, nu=0.01))
    oc.update_fields()
    for c in range(3):
        oc.assemble_u(c); oc.solve(0); oc.correct_u(c)
    oc.assemble_p()
    systems.append((oc.mesh.get("rowptr"), oc.mesh.get("col"), oc.get("ac"), oc.get("anb"), oc.get("bc")))
    # one call on a small system first, so that loading the entry point's kernels (which takes
    # device memory for their code) happens before the calls whose memory use is checked
    rp_w, col_w, ac_w, anb_w, bc_w = random_diag_dominant(64, 3, nbr=4)
    w = _system(torch, rp_w, col_w, ac_w, anb_w, bc_w, np.zeros(64))
    assert _call(lib, "ufvm_solve_sor_noalloc", 64, w, stream) == 0, lib.ufvm_last_error()
    torch.cuda.synchronize()
    for k, (rp, col, ac, anb, bc) in enumerate(systems):
        n = len(ac)
        x0 = rng.normal(size=n)
        a = _system(torch, rp, col, ac, anb, bc, x0)
        b = [t.clone() for t in a]
        assert _call(lib, "ufvm_solve_sor", n, a, stream) == 0, lib.ufvm_last_error()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        assert _call(lib, "ufvm_solve_sor_noalloc", n, b, stream) == 0, lib.ufvm_last_error()
        torch.cuda.synchronize()
        # the call alone took no device memory
        assert torch.cuda.mem_get_info()[0] == free_before, f"call {k} changed the free device memory"
        xa, xb = a[5].cpu().numpy(), b[5].cpu().numpy()
        assert np.array_equal(xa, xb), f"call {k}: max |d| = {np.abs(xa - xb).max():.3e}"
        assert not np.array_equal(xb, x0)


@pytest.mark.gpu
def test_noalloc_sor_rejects_oversized_systems(ufvm_mod):
    import torch
    lib = ufvm_mod.lib()
    n = MAX_ROWS + 1
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = ct.c_void_p(dummy.data_ptr())
    code = lib.ufvm_solve_sor_noalloc(n, p, p, p, p, p, p, ct.c_void_p(0))
    assert code != 0
    assert b"262144" in lib.ufvm_last_error()
