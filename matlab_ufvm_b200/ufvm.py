"""Host-side mirror of uFVM's function interface for the steady SIMPLE path, over libufvm.so.

uFVM binds functions by MATLAB path and keeps all state in the global ``Domain`` struct
(``setup/cfdSetupDomain.m:11-63``). Here the state is a device-resident case handle, and
the functions keep the reference's names, argument meaning and error behaviour:

==================================  ==========================================================
reference (uFVM/src/...)            here
==================================  ==========================================================
``cfdUpdateFields``                 :meth:`GpuCase.cfdUpdateFields`
``cfdAssembleEquation(name, i)``    :meth:`GpuCase.cfdAssembleEquation` -> (rms, max)
``cfdSolveEquation(name)``          :meth:`GpuCase.cfdSolveEquation` -> (r0, r1)
``cfdCorrectEquation(name, i)``     :meth:`GpuCase.cfdCorrectEquation`
``cfdAssembleAndCorrectEquation``   :meth:`GpuCase.cfdAssembleAndCorrectEquation`
``cfdRunCase`` (steady branch)      :meth:`GpuCase.cfdRunCase`
``cfdComputeResidualsArray``        :func:`cfdComputeResidualsArray`
``cfdSolveSOR``                     :func:`cfdSolveSOR`
``cfdFactorizeILU / cfdSolveILU``   :func:`cfdFactorizeILU`, :func:`cfdSolveILU`
``cfdSolveAlgebraicSystem``         :func:`cfdSolveAlgebraicSystem`
``cfdAgglomerateLevel``             :func:`cfdAgglomerateLevel`
==================================  ==========================================================

Errors raise :class:`UfvmError` carrying the library's status code and message, the
counterpart of the reference's ``error('...')`` calls. There is no CPU fallback: if
libufvm.so is missing or no GPU is present, calls raise.
"""
from __future__ import annotations

import ctypes as ct
import os
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import case as _case

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libufvm.so")

STATUS = {0: "UFVM_OK", 1: "UFVM_E_INVALID", 2: "UFVM_E_CUDA", 3: "UFVM_E_OOM", 4: "UFVM_E_NAN",
          5: "UFVM_E_ZERO_DIAG", 6: "UFVM_E_BC_UNSUPPORTED", 7: "UFVM_E_AMG_LEVELS", 8: "UFVM_E_TIMEOUT",
          9: "UFVM_E_NOT_CONVERGED"}
EQ = {"U": 0, "p": 1}


class UfvmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class MeshDesc(ct.Structure):
    _fields_ = [("n_points", ct.c_int32), ("points", ct.POINTER(ct.c_double)),
                ("n_faces", ct.c_int32), ("face_start", ct.POINTER(ct.c_int32)),
                ("face_nodes", ct.POINTER(ct.c_int32)), ("n_interior", ct.c_int32),
                ("owner", ct.POINTER(ct.c_int32)), ("neighbour", ct.POINTER(ct.c_int32)),
                ("n_patches", ct.c_int32), ("patch_type", ct.POINTER(ct.c_int32)),
                ("patch_start", ct.POINTER(ct.c_int32)), ("patch_n", ct.POINTER(ct.c_int32))]


class Settings(ct.Structure):
    _fields_ = [(n, ct.c_int32) for n in (
        "n_correctors", "fixed_element", "p_cycle", "p_max_cycles", "p_max_coarse_levels", "p_pre_sweep",
        "p_post_sweep", "p_smoother", "u_smoother", "u_n_iter", "quirks", "p_amg", "precision",
        "hierarchy_reuse", "p_krylov", "service_eager")] + [(n, ct.c_double) for n in (
            "nu", "urf_u", "urf_p", "tol_u", "tol_p", "p_termination", "u_rrf", "false_dt", "p_coarse_weight")]


_lib = None
D = ct.POINTER(ct.c_double)
I32 = ct.POINTER(ct.c_int32)
VP = ct.c_void_p


def lib():
    """Load libufvm.so (in-tree build). Raises if it is missing: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise UfvmError(2, f"{LIB_PATH} not built (run python -m matlab_ufvm_b200.build)")
    L = ct.CDLL(LIB_PATH)
    L.ufvm_last_error.restype = ct.c_char_p
    L.ufvm_version.restype = ct.c_char_p
    L.ufvm_case_create.argtypes = [ct.POINTER(MeshDesc), ct.POINTER(Settings), I32, I32, D, D, D, D, D,
                                   ct.POINTER(VP)]
    L.ufvm_case_destroy.argtypes = [VP]
    L.ufvm_case_sizes.argtypes = [VP, ct.POINTER(ct.c_int64)]
    L.ufvm_update_fields.argtypes = [VP]
    L.ufvm_assemble_equation.argtypes = [VP, ct.c_int, ct.c_int, D, D]
    L.ufvm_solve_equation.argtypes = [VP, ct.c_int, D, D]
    L.ufvm_correct_equation.argtypes = [VP, ct.c_int, ct.c_int]
    L.ufvm_simple_iteration.argtypes = [VP, D, ct.POINTER(ct.c_int)]
    L.ufvm_run_case.argtypes = [VP, ct.c_int, ct.POINTER(ct.c_int), D]
    L.ufvm_get_field.argtypes = [VP, ct.c_char_p, D, ct.c_int64, ct.POINTER(ct.c_int64)]
    L.ufvm_set_field.argtypes = [VP, ct.c_char_p, D, ct.c_int64]
    L.ufvm_get_geometry.argtypes = [VP, ct.c_char_p, D, ct.c_int64]
    L.ufvm_get_levels.argtypes = [VP, ct.POINTER(ct.c_int), ct.POINTER(ct.c_int64), ct.c_int]
    L.ufvm_get_level_array.argtypes = [VP, ct.c_int, ct.c_char_p, VP, ct.c_int64, ct.POINTER(ct.c_int64)]
    for name, extra in (("ufvm_compute_residuals_array", [VP, VP, VP, VP, VP, VP, VP, VP]),
                        ("ufvm_solve_sor", [VP, VP, VP, VP, VP, VP, VP]),
                        ("ufvm_solve_sor_noalloc", [VP, VP, VP, VP, VP, VP, VP]),
                        ("ufvm_solve_ilu", [VP, VP, VP, VP, VP, VP, VP, VP])):
        getattr(L, name).argtypes = [ct.c_int32] + extra
    L.ufvm_factorize_ilu.argtypes = [ct.c_int32, VP, VP, VP, VP, VP, ct.c_int32, VP]
    L.ufvm_solve_algebraic_system.argtypes = [ct.c_int32, VP, VP, VP, VP, VP, VP, ct.c_int32, ct.c_int32,
                                              ct.c_double, ct.c_int32, D, D, I32, VP]
    L.ufvm_agglomerate_level.argtypes = [ct.c_int32, VP, VP, VP, VP, VP, VP, VP, VP, VP, I32, I32, VP]
    L.ufvm_profile_plain_kernel.argtypes = [ct.c_int32, ct.c_int32, VP, VP, VP, VP, VP, VP, ct.c_int32, D, D, VP]
    _lib = L
    return L


def _check(code: int):
    if code != 0:
        raise UfvmError(code, lib().ufvm_last_error().decode())


def _dp(a):
    return None if a is None else a.ctypes.data_as(D)


def _ip(a):
    return a.ctypes.data_as(I32)


def settings_from_spec(spec: _case.CaseSpec, precision: int = 0, hierarchy_reuse: int = 0) -> Settings:
    s = Settings()
    iv = spec.iset()
    for k, n in enumerate(("n_correctors", "fixed_element", "p_cycle", "p_max_cycles", "p_max_coarse_levels",
                           "p_pre_sweep", "p_post_sweep", "p_smoother", "u_smoother", "u_n_iter", "quirks",
                           "p_amg")):
        setattr(s, n, int(iv[k]))
    s.precision = precision
    s.hierarchy_reuse = hierarchy_reuse
    dv = spec.dset()
    for k, n in enumerate(("nu", "urf_u", "urf_p", "tol_u", "tol_p", "p_termination", "u_rrf", "false_dt")):
        setattr(s, n, float(dv[k]))
    return s


class GpuCase:
    """One device-resident steady case (the GPU counterpart of the global ``Domain``)."""

    def __init__(self, spec: _case.CaseSpec, precision: int = 0, hierarchy_reuse: int = 0):
        L = lib()
        m = spec.mesh
        self.spec = spec
        self._keep = k = dict(
            pts=np.ascontiguousarray(m.points, dtype=np.float64),
            fs=np.ascontiguousarray(m.face_start, dtype=np.int32),
            fn=np.ascontiguousarray(m.face_nodes, dtype=np.int32),
            own=np.ascontiguousarray(m.owner, dtype=np.int32),
            nei=np.ascontiguousarray(m.neighbour, dtype=np.int32),
            pt=spec.patch_types(),
            ps=np.array([p.start for p in m.patches], dtype=np.int32),
            pn=np.array([p.n for p in m.patches], dtype=np.int32))
        md = MeshDesc(k["pts"].shape[0], _dp(k["pts"]), k["own"].shape[0], _ip(k["fs"]), _ip(k["fn"]),
                      k["nei"].shape[0], _ip(k["own"]), _ip(k["nei"]), len(m.patches), _ip(k["pt"]),
                      _ip(k["ps"]), _ip(k["pn"]))
        self.settings = settings_from_spec(spec, precision, hierarchy_reuse)
        bu, bp = spec.bc_codes()
        vu = np.ascontiguousarray(spec.val_u, dtype=np.float64)
        vp = np.ascontiguousarray(spec.val_p, dtype=np.float64)
        U0 = None if spec.U0 is None else np.ascontiguousarray(spec.U0, dtype=np.float64)
        p0 = None if spec.p0 is None else np.ascontiguousarray(spec.p0, dtype=np.float64)
        m0 = None if spec.mdot0 is None else np.ascontiguousarray(spec.mdot0, dtype=np.float64)
        self._keep.update(bu=bu, bp=bp, vu=vu, vp=vp, U0=U0, p0=p0, m0=m0)
        h = VP()
        _check(L.ufvm_case_create(ct.byref(md), ct.byref(self.settings), _ip(bu), _ip(bp), _dp(vu), _dp(vp),
                                  _dp(U0), _dp(p0), _dp(m0), ct.byref(h)))
        self.h = h
        sz = (ct.c_int64 * 4)()
        _check(L.ufvm_case_sizes(self.h, sz))
        self.Nc, self.F, self.Fi, self.nnz = (int(x) for x in sz)
        self.Fb = self.F - self.Fi

    def close(self):
        if getattr(self, "h", None):
            lib().ufvm_case_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- reference-named entry points
    def cfdUpdateFields(self):
        _check(lib().ufvm_update_fields(self.h))

    def cfdAssembleEquation(self, name: str, iComponent: int = 1) -> Tuple[float, float]:
        r, m = ct.c_double(), ct.c_double()
        _check(lib().ufvm_assemble_equation(self.h, EQ[name], iComponent - 1, ct.byref(r), ct.byref(m)))
        return r.value, m.value

    def cfdSolveEquation(self, name: str) -> Tuple[float, float]:
        r0, r1 = ct.c_double(), ct.c_double()
        _check(lib().ufvm_solve_equation(self.h, EQ[name], ct.byref(r0), ct.byref(r1)))
        return r0.value, r1.value

    def cfdCorrectEquation(self, name: str, iComponent: int = 1):
        _check(lib().ufvm_correct_equation(self.h, EQ[name], iComponent - 1))

    def cfdAssembleAndCorrectEquation(self, name: str):
        """assemble/cfdAssembleAndCorrectEquation.m:35-49 -> (rms, max, r0, r1) per component."""
        ncomp = 3 if name == "U" else 1
        ncorr = self.spec.n_correctors if name == "p" else 1
        out = np.zeros((4, ncomp))
        for c in range(ncomp):
            for _ in range(ncorr):
                out[0, c], out[1, c] = self.cfdAssembleEquation(name, c + 1)
                out[2, c], out[3, c] = self.cfdSolveEquation(name)
                self.cfdCorrectEquation(name, c + 1)
        return out

    def iterate(self) -> Tuple[np.ndarray, bool]:
        res = np.zeros(16)
        conv = ct.c_int()
        _check(lib().ufvm_simple_iteration(self.h, _dp(res), ct.byref(conv)))
        return res, bool(conv.value)

    def cfdRunCase(self, max_iter: int = 10000) -> Tuple[int, np.ndarray]:
        """Steady branch of top/cfdRunCase.m: iterate to residualControl; raises on NaN."""
        res = np.zeros(16)
        it = ct.c_int()
        code = lib().ufvm_run_case(self.h, max_iter, ct.byref(it), _dp(res))
        if code not in (0, 9):
            _check(code)
        return it.value, res

    # ---- field access
    def get(self, name: str) -> np.ndarray:
        n = ct.c_int64()
        _check(lib().ufvm_get_field(self.h, name.encode(), None, 0, ct.byref(n)))
        out = np.zeros(n.value)
        _check(lib().ufvm_get_field(self.h, name.encode(), _dp(out), n.value, ct.byref(n)))
        return out

    def set(self, name: str, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        _check(lib().ufvm_set_field(self.h, name.encode(), _dp(a), a.size))

    def geometry(self, name: str) -> np.ndarray:
        vec = name in ("Sf", "centroid_f", "CN", "eCN", "T", "centroid_c")
        n = self.Nc if name in ("volume", "centroid_c") else self.F
        out = np.zeros((n, 3) if vec else n)
        _check(lib().ufvm_get_geometry(self.h, name.encode(), _dp(out), out.size))
        return out

    def levels(self):
        nl = ct.c_int()
        sizes = (ct.c_int64 * 16)()
        _check(lib().ufvm_get_levels(self.h, ct.byref(nl), sizes, 16))
        return [int(sizes[i]) for i in range(nl.value)]

    def level_array(self, level: int, name: str) -> np.ndarray:
        n = ct.c_int64()
        _check(lib().ufvm_get_level_array(self.h, level, name.encode(), None, 0, ct.byref(n)))
        dt = np.float64 if name in ("ac", "anb") else np.int32
        out = np.zeros(n.value, dtype=dt)
        _check(lib().ufvm_get_level_array(self.h, level, name.encode(), out.ctypes.data_as(VP), n.value,
                                          ct.byref(n)))
        return out


# ---------------------------------------------------------------- matrix-level functions
def _dev(x, dtype):
    import torch
    t = torch.as_tensor(np.ascontiguousarray(x, dtype=dtype)).cuda()
    return t


def _ptr(t):
    return ct.c_void_p(t.data_ptr())


def _coeffs_to_dev(rowptr, col, ac, anb, bc, dphi):
    import torch
    return (_dev(rowptr, np.int32), _dev(col, np.int32), _dev(ac, np.float64), _dev(anb, np.float64),
            _dev(bc, np.float64), _dev(dphi, np.float64))


def _stream():
    import torch
    return ct.c_void_p(torch.cuda.current_stream().cuda_stream)


def cfdComputeResidualsArray(rowptr, col, ac, anb, bc, dphi) -> np.ndarray:
    """compute/cfdComputeResidualsArray.m:9-17 on the GPU (host arrays in, host array out)."""
    import torch
    rp, cl, a, b, c, x = _coeffs_to_dev(rowptr, col, ac, anb, bc, dphi)
    r = torch.empty_like(a)
    _check(lib().ufvm_compute_residuals_array(len(ac), _ptr(rp), _ptr(cl), _ptr(a), _ptr(b), _ptr(c), _ptr(x),
                                              _ptr(r), _stream()))
    torch.cuda.synchronize()
    return r.cpu().numpy()


def cfdSolveSOR(rowptr, col, ac, anb, bc, dphi) -> np.ndarray:
    """solve/cfdSolveSOR.m:13-29: one symmetric natural-order Gauss-Seidel sweep."""
    import torch
    rp, cl, a, b, c, x = _coeffs_to_dev(rowptr, col, ac, anb, bc, dphi)
    _check(lib().ufvm_solve_sor(len(ac), _ptr(rp), _ptr(cl), _ptr(a), _ptr(b), _ptr(c), _ptr(x), _stream()))
    torch.cuda.synchronize()
    return x.cpu().numpy()


def cfdFactorizeILU(rowptr, col, ac, anb, quirks: int = _case.QUIRKS_REFERENCE) -> np.ndarray:
    """solve/cfdFactorizeILU.m:5-47 -> dc (inverted DILU diagonal)."""
    import torch
    rp, cl, a, b = _dev(rowptr, np.int32), _dev(col, np.int32), _dev(ac, np.float64), _dev(anb, np.float64)
    dc = torch.empty_like(a)
    _check(lib().ufvm_factorize_ilu(len(ac), _ptr(rp), _ptr(cl), _ptr(a), _ptr(b), _ptr(dc), int(quirks), _stream()))
    torch.cuda.synchronize()
    return dc.cpu().numpy()


def cfdSolveILU(rowptr, col, ac, anb, bc, dc, dphi) -> np.ndarray:
    """solve/cfdSolveILU.m:18-93: one DILU application, returns the updated dphi."""
    import torch
    rp, cl, a, b, c, x = _coeffs_to_dev(rowptr, col, ac, anb, bc, dphi)
    d = _dev(dc, np.float64)
    _check(lib().ufvm_solve_ilu(len(ac), _ptr(rp), _ptr(cl), _ptr(a), _ptr(b), _ptr(c), _ptr(d), _ptr(x), _stream()))
    torch.cuda.synchronize()
    return x.cpu().numpy()


def cfdSolveAlgebraicSystem(rowptr, col, ac, anb, bc, dphi, smoother: str = "ILU", nIter: int = 10,
                            rrf: float = 0.1, quirks: int = _case.QUIRKS_REFERENCE):
    """solve/cfdSolveAlgebraicSystem.m:11-66 -> (dphi, r0, r1, iterations)."""
    import torch
    rp, cl, a, b, c, x = _coeffs_to_dev(rowptr, col, ac, anb, bc, dphi)
    r0, r1, it = ct.c_double(), ct.c_double(), ct.c_int32()
    _check(lib().ufvm_solve_algebraic_system(len(ac), _ptr(rp), _ptr(cl), _ptr(a), _ptr(b), _ptr(c), _ptr(x),
                                             _case.SMOOTHER[smoother], nIter, rrf, int(quirks), ct.byref(r0),
                                             ct.byref(r1), ct.byref(it), _stream()))
    torch.cuda.synchronize()
    return x.cpu().numpy(), r0.value, r1.value, it.value


PLAIN_KERNELS = {"residual": 0, "SOR": 1, "MCGS": 2, "ILU": 3}


def profile_plain_kernel(kernel: str, rowptr, col, ac, anb, bc, dphi, reps: int = 5):
    """Kernel time of one stand-alone solver kernel on DEVICE tensors (the plain form's roofline
    measurement): "residual", "SOR" (level-scheduled natural-order sweep), "MCGS" (multicolour
    sweep) or "ILU" (one DILU application). L2 is flushed (by reads) before every timed launch.
    Returns (ms per launch, algorithmic bytes per launch). Sweeps overwrite dphi."""
    ms, by = ct.c_double(), ct.c_double()
    _check(lib().ufvm_profile_plain_kernel(PLAIN_KERNELS[kernel], len(ac), _ptr(rowptr), _ptr(col), _ptr(ac),
                                           _ptr(anb), _ptr(bc), _ptr(dphi), int(reps), ct.byref(ms), ct.byref(by),
                                           _stream()))
    return ms.value, by.value


def cfdAgglomerateLevel(rowptr, col, ac, anb):
    """solve/AMG/cfdAgglomerateLevel.m + assembleAgglomeratedLHS.m on the GPU.

    Returns (parents 0-based, coarse rowptr, coarse col, coarse ac, coarse anb)."""
    import torch
    n = len(ac)
    nnz = int(rowptr[-1])
    rp, cl, a, b = _dev(rowptr, np.int32), _dev(col, np.int32), _dev(ac, np.float64), _dev(anb, np.float64)
    par = torch.empty(n, dtype=torch.int32, device="cuda")
    crp = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    ccol = torch.empty(max(nnz, 1), dtype=torch.int32, device="cuda")
    cac = torch.empty(n, dtype=torch.float64, device="cuda")
    canb = torch.empty(max(nnz, 1), dtype=torch.float64, device="cuda")
    nc, cnnz = ct.c_int32(), ct.c_int32()
    _check(lib().ufvm_agglomerate_level(n, _ptr(rp), _ptr(cl), _ptr(a), _ptr(b), _ptr(par), _ptr(crp), _ptr(ccol),
                                        _ptr(cac), _ptr(canb), ct.byref(nc), ct.byref(cnnz), _stream()))
    torch.cuda.synchronize()
    k, q = nc.value, cnnz.value
    return (par.cpu().numpy(), crp[:k + 1].cpu().numpy(), ccol[:q].cpu().numpy(), cac[:k].cpu().numpy(),
            canb[:q].cpu().numpy())


# ---------------------------------------------------------------- batched service
def _service_lib():
    L = lib()
    if not getattr(L, "_svc_ready", False):
        L.ufvm_service_create.argtypes = [ct.POINTER(Settings), ct.c_int64, ct.POINTER(VP)]
        L.ufvm_service_submit.argtypes = [VP, ct.POINTER(MeshDesc), ct.c_double, I32, I32, D, D, ct.c_int32,
                                          ct.POINTER(ct.c_int64)]
        L.ufvm_service_step.argtypes = [VP, ct.POINTER(ct.c_int32), ct.POINTER(ct.c_int32), ct.POINTER(ct.c_int64)]
        L.ufvm_service_status.argtypes = [VP, ct.c_int64, ct.POINTER(ct.c_int32), ct.POINTER(ct.c_int32),
                                          ct.POINTER(ct.c_int32), D, D, D]
        L.ufvm_service_get_field.argtypes = [VP, ct.c_int64, ct.c_char_p, D, ct.c_int64, ct.POINTER(ct.c_int64)]
        L.ufvm_service_release.argtypes = [VP, ct.c_int64]
        L.ufvm_service_destroy.argtypes = [VP]
        L.ufvm_service_stats.argtypes = [VP, D, ct.c_int]
        L.ufvm_service_stream.argtypes = [VP, ct.POINTER(VP)]
        L.ufvm_service_profile.argtypes = [VP, ct.c_int32, ct.c_int32, D, D]
        L.ufvm_service_poll.argtypes = [VP, ct.POINTER(ct.c_int64), ct.c_int64, ct.POINTER(ct.c_int64)]
        L.ufvm_service_set_admit_interval.argtypes = [VP, ct.c_int32]
        L.ufvm_service_set_schedule.argtypes = [VP, ct.c_int32, ct.c_int32]
        L.ufvm_service_set_memory_budget.argtypes = [VP, ct.c_int64]
        L.ufvm_service_admit.argtypes = [VP, ct.POINTER(ct.c_int32)]
        L.ufvm_service_inject_admit_oom.argtypes = [VP, ct.c_int64, ct.c_int32]
        L._svc_ready = True
    return L


def fast_settings(spec: _case.CaseSpec, hierarchy_reuse: int = 1000000, p_krylov: int = 1) -> Settings:
    """Service settings: the case's SIMPLE settings with multicolour GS and FP32 AMG
    (p_krylov 1: the FP32 V-cycle, one pre- and one post-smoothing sweep, preconditions a
    flexible CG in FP64)."""
    s = settings_from_spec(spec, precision=1, hierarchy_reuse=hierarchy_reuse)
    s.p_krylov = p_krylov
    # one post-smoothing sweep: the flexible CG recovers the convergence of the reference's
    # three, and each V-cycle costs about 40% less on level 0
    s.p_post_sweep = 1
    # over-correction of the piecewise-constant prolongation: doubling the coarse-grid correction
    # cuts the flexible-CG iterations per p solve about threefold on the cavity sweep
    s.p_coarse_weight = 2.0
    s.p_smoother = _case.SMOOTHER["MCGS"]
    s.u_smoother = _case.SMOOTHER["MCGS"]
    s.p_cycle = _case.CYCLE["V-Cycle"]
    return s


class Service:
    """Continuous-batching steady-case service (ufvm_service_* in include/ufvm.h)."""

    STATES = {0: "queued", 1: "resident", 2: "converged", 3: "stopped"}

    def __init__(self, settings: Settings, max_resident_cells: int = 8_000_000):
        L = _service_lib()
        self.settings = settings
        h = VP()
        _check(L.ufvm_service_create(ct.byref(settings), int(max_resident_cells), ct.byref(h)))
        self.h = h
        self._specs = {}

    def submit(self, spec: _case.CaseSpec, max_iter: int = 5000) -> int:
        L = _service_lib()
        m = spec.mesh
        k = dict(pts=np.ascontiguousarray(m.points, dtype=np.float64),
                 fs=np.ascontiguousarray(m.face_start, dtype=np.int32),
                 fn=np.ascontiguousarray(m.face_nodes, dtype=np.int32),
                 own=np.ascontiguousarray(m.owner, dtype=np.int32),
                 nei=np.ascontiguousarray(m.neighbour, dtype=np.int32), pt=spec.patch_types(),
                 ps=np.array([p.start for p in m.patches], dtype=np.int32),
                 pn=np.array([p.n for p in m.patches], dtype=np.int32))
        md = MeshDesc(k["pts"].shape[0], _dp(k["pts"]), k["own"].shape[0], _ip(k["fs"]), _ip(k["fn"]),
                      k["nei"].shape[0], _ip(k["own"]), _ip(k["nei"]), len(m.patches), _ip(k["pt"]),
                      _ip(k["ps"]), _ip(k["pn"]))
        bu, bp = spec.bc_codes()
        vu = np.ascontiguousarray(spec.val_u, dtype=np.float64)
        vp = np.ascontiguousarray(spec.val_p, dtype=np.float64)
        t = ct.c_int64()
        _check(L.ufvm_service_submit(self.h, ct.byref(md), float(spec.nu), _ip(bu), _ip(bp), _dp(vu), _dp(vp),
                                     int(max_iter), ct.byref(t)))
        self._specs[t.value] = spec
        return t.value

    def step(self):
        nr, nq, nf = ct.c_int32(), ct.c_int32(), ct.c_int64()
        _check(_service_lib().ufvm_service_step(self.h, ct.byref(nr), ct.byref(nq), ct.byref(nf)))
        return nr.value, nq.value, nf.value

    def status(self, ticket: int) -> Dict:
        st, code, it = ct.c_int32(), ct.c_int32(), ct.c_int32()
        res = np.zeros(16)
        lat, qu = ct.c_double(), ct.c_double()
        _check(_service_lib().ufvm_service_status(self.h, ticket, ct.byref(st), ct.byref(code), ct.byref(it),
                                                  _dp(res), ct.byref(lat), ct.byref(qu)))
        return dict(state=self.STATES[st.value], status=code.value, iterations=it.value, res=res,
                    latency_ms=lat.value, queue_ms=qu.value)

    def field(self, ticket: int, name: str) -> np.ndarray:
        L = _service_lib()
        n = ct.c_int64()
        _check(L.ufvm_service_get_field(self.h, ticket, name.encode(), None, 0, ct.byref(n)))
        out = np.zeros(n.value)
        _check(L.ufvm_service_get_field(self.h, ticket, name.encode(), _dp(out), n.value, ct.byref(n)))
        return out

    PHASES = ("update", "assemble_u", "solve_u", "correct_u", "assemble_p", "hierarchy", "solve_p", "correct_p")

    def stats(self) -> Dict:
        out = np.zeros(34)
        _check(_service_lib().ufvm_service_stats(self.h, _dp(out), 34))
        d = {f"{k}_ms": float(out[i]) for i, k in enumerate(self.PHASES)}
        d.update(u_sweeps=int(out[8]), p_cycles=int(out[9]), steps=int(out[10]), clock_ms=float(out[11]),
                 graph_ticks=int(out[12]), captures=int(out[13]), graph_launches=int(out[14]),
                 cta_rows=int(out[15]), tunes=int(out[16]), resident_bytes=int(out[17]),
                 memory_budget=int(out[18]), deferred_for_memory=int(out[19]), oom_requeues=int(out[20]),
                 slot_drops=int(out[21]), footprint_scale=float(out[22]), u_loop_bodies=int(out[23]),
                 p_loop_bodies=int(out[24]), host_rebuild_ms=float(out[25]), host_capture_ms=float(out[26]),
                 host_drop_ms=float(out[27]), build_wall_ms=float(out[28]), build_agg_ms=float(out[29]),
                 build_color_ms=float(out[30]), build_ell_ms=float(out[31]), build_alloc_ms=float(out[32]),
                 host_admit_ms=float(out[33]))
        return d

    def admit(self) -> int:
        """Admit queued cases now (uploads and processes their meshes); returns the active cases."""
        n = ct.c_int32()
        _check(_service_lib().ufvm_service_admit(self.h, ct.byref(n)))
        return n.value

    def inject_admit_oom(self, ticket: int, count: int = 1):
        """Test hook: the next `count` admissions of `ticket` fail as an out-of-memory."""
        _check(_service_lib().ufvm_service_inject_admit_oom(self.h, int(ticket), int(count)))

    def set_memory_budget(self, nbytes: int):
        """HBM budget (bytes) that admission keeps the resident cases and unreleased results in."""
        _check(_service_lib().ufvm_service_set_memory_budget(self.h, int(nbytes)))

    def poll(self, capacity: int = 4096) -> List[int]:
        """Tickets finished since the previous poll."""
        buf = (ct.c_int64 * capacity)()
        n = ct.c_int64()
        _check(_service_lib().ufvm_service_poll(self.h, buf, capacity, ct.byref(n)))
        return [int(buf[i]) for i in range(n.value)]

    def set_schedule(self, cta_rows: int, packed: int = 1):
        """Fix the V-cycle's launch schedule (cta_rows 0: back to the autotuner)."""
        _check(_service_lib().ufvm_service_set_schedule(self.h, int(cta_rows), int(packed)))

    def set_admit_interval(self, steps: int):
        _check(_service_lib().ufvm_service_set_admit_interval(self.h, int(steps)))

    def stream(self) -> int:
        """The cudaStream_t (as an integer) that all of the service's device work runs on."""
        v = VP()
        _check(_service_lib().ufvm_service_stream(self.h, ct.byref(v)))
        return int(v.value or 0)

    def profile(self, kernel: int, reps: int = 20) -> Tuple[float, float]:
        """(ms per unit, compulsory bytes per unit) of one tick kernel on the resident batch."""
        ms, by = ct.c_double(), ct.c_double()
        _check(_service_lib().ufvm_service_profile(self.h, int(kernel), int(reps), ct.byref(ms), ct.byref(by)))
        return ms.value, by.value

    def release(self, ticket: int):
        _check(_service_lib().ufvm_service_release(self.h, ticket))
        self._specs.pop(ticket, None)

    def run(self, max_steps: int = 100000):
        """Step until nothing is resident or queued; returns the number of steps."""
        steps = 0
        while steps < max_steps:
            nr, nq, _ = self.step()
            steps += 1
            if nr == 0 and nq == 0:
                break
        return steps

    def close(self):
        if getattr(self, "h", None):
            _service_lib().ufvm_service_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
