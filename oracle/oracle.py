"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg to check or
time the CUDA library against a single-thread restatement of the reference. Nothing in
the product package imports this module.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libufvm_oracle.so")
_lib = None

D = ct.POINTER(ct.c_double)
I = ct.POINTER(ct.c_int)
V = ct.c_void_p


def build(force: bool = False) -> str:
    if force or not os.path.exists(_LIB_PATH) or \
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "ufvm_oracle.cpp")):
        subprocess.run(["make", "-C", _HERE], check=True, capture_output=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ct.CDLL(_LIB_PATH)
        L.orc_mesh_create.restype = V
        L.orc_mesh_create.argtypes = [ct.c_int, D, ct.c_int, I, I, ct.c_int, I, I, ct.c_int, I, I, I, ct.c_int]
        L.orc_mesh_destroy.argtypes = [V]
        L.orc_mesh_sizes.argtypes = [V, I]
        L.orc_mesh_get.argtypes = [V, ct.c_char_p, V]
        L.orc_case_create.restype = V
        L.orc_case_create.argtypes = [V, I, D, I, I, D, D, D, D, D]
        L.orc_case_destroy.argtypes = [V]
        L.orc_case_iterate.argtypes = [V, D]
        L.orc_update_fields.argtypes = [V]
        L.orc_assemble_u.argtypes = [V, ct.c_int, D, D]
        L.orc_assemble_p.argtypes = [V, D, D]
        L.orc_solve.argtypes = [V, ct.c_int, D, D]
        L.orc_correct_u.argtypes = [V, ct.c_int]
        L.orc_correct_p.argtypes = [V]
        L.orc_case_get.argtypes = [V, ct.c_char_p, D, I]
        L.orc_case_set.argtypes = [V, ct.c_char_p, D]
        L.orc_case_nlevels.argtypes = [V]
        L.orc_level_get.argtypes = [V, ct.c_int, ct.c_char_p, V, I]
        L.orc_residuals.argtypes = [ct.c_int, I, I, D, D, D, D, D]
        L.orc_sor_sweep.argtypes = [ct.c_int, I, I, D, D, D, D]
        L.orc_ilu_factor.argtypes = [ct.c_int, I, I, D, D, D, ct.c_int]
        L.orc_ilu_sweep.argtypes = [ct.c_int, I, I, D, D, D, D, D]
        L.orc_mcgs_sweep.argtypes = [ct.c_int, I, I, D, D, D, I, ct.c_int, D]
        L.orc_coloring.argtypes = [ct.c_int, I, I, I]
        L.orc_solve_algebraic_system.argtypes = [ct.c_int, I, I, D, D, D, D, ct.c_int, ct.c_int, ct.c_double,
                                                 ct.c_int, D, D, I]
        L.orc_agglomerate.argtypes = [ct.c_int, I, I, D, D, I, I, I, D, D, I]
        _lib = L
    return _lib


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def dp(a):
    return a.ctypes.data_as(D) if a is not None else None


def ip(a):
    return a.ctypes.data_as(I) if a is not None else None


class OracleMesh:
    def __init__(self, mesh, quirks: int):
        L = lib()
        self._keep = [_d(mesh.points), _i(mesh.face_start), _i(mesh.face_nodes), _i(mesh.owner),
                      _i(mesh.neighbour)]
        from matlab_ufvm_b200.case import PHYS
        pt = _i([PHYS[p.type] for p in mesh.patches])
        ps = _i([p.start for p in mesh.patches])
        pn = _i([p.n for p in mesh.patches])
        self._keep += [pt, ps, pn]
        pts, fs, fn, own, nei = self._keep[:5]
        self.h = L.orc_mesh_create(pts.shape[0], dp(pts), own.shape[0], ip(fs), ip(fn), nei.shape[0], ip(own),
                                   ip(nei), len(mesh.patches), ip(pt), ip(ps), ip(pn), int(quirks))
        s = np.zeros(4, dtype=np.int32)
        L.orc_mesh_sizes(self.h, ip(s))
        self.Nc, self.F, self.Fi, self.nnz = (int(x) for x in s)

    _VEC = {"Sf", "centroid_f", "CN", "eCN", "T"}
    _SIZE = {"area": "F", "gDiff": "F", "gf": "F", "walldist": "F", "volume": "Nc", "centroid_c": "Nc3"}

    def get(self, name):
        L = lib()
        if name in self._VEC:
            out = np.zeros((self.F, 3))
        elif name == "centroid_c":
            out = np.zeros((self.Nc, 3))
        elif name in ("area", "gDiff", "gf", "walldist"):
            out = np.zeros(self.F)
        elif name == "volume":
            out = np.zeros(self.Nc)
        elif name == "rowptr":
            out = np.zeros(self.Nc + 1, dtype=np.int32)
        elif name == "col":
            out = np.zeros(self.nnz, dtype=np.int32)
        elif name in ("own_slot", "nei_slot"):
            out = np.zeros(self.Fi, dtype=np.int32)
        elif name == "cell_face_start":
            out = np.zeros(self.Nc + 1, dtype=np.int32)
        elif name == "cell_faces":
            out = np.zeros(self.F + self.Fi, dtype=np.int32)
        else:
            raise KeyError(name)
        rc = L.orc_mesh_get(self.h, name.encode(), out.ctypes.data_as(V))
        assert rc >= 0, name
        return out

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_mesh_destroy(self.h)
            self.h = None


class OracleCase:
    """The reference's SIMPLE driver restated on the CPU (cfdRunCase steady branch)."""

    def __init__(self, spec):
        L = lib()
        self.spec = spec
        self.mesh = OracleMesh(spec.mesh, spec.quirks)
        bu, bp = spec.bc_codes()
        self._keep = [spec.iset(), spec.dset(), bu, bp, _d(spec.val_u), _d(spec.val_p),
                      None if spec.U0 is None else _d(spec.U0), None if spec.p0 is None else _d(spec.p0),
                      None if spec.mdot0 is None else _d(spec.mdot0)]
        k = self._keep
        self.h = L.orc_case_create(self.mesh.h, ip(k[0]), dp(k[1]), ip(k[2]), ip(k[3]), dp(k[4]), dp(k[5]),
                                   dp(k[6]), dp(k[7]), dp(k[8]))
        self.Nc, self.F, self.Fi = self.mesh.Nc, self.mesh.F, self.mesh.Fi
        self.Fb = self.F - self.Fi

    def iterate(self):
        res = np.zeros(16)
        rc = lib().orc_case_iterate(self.h, dp(res))
        return rc, res

    def update_fields(self):
        lib().orc_update_fields(self.h)

    def assemble_u(self, comp):
        r, m = ct.c_double(), ct.c_double()
        rc = lib().orc_assemble_u(self.h, comp, ct.byref(r), ct.byref(m))
        assert rc == 0, rc
        return r.value, m.value

    def assemble_p(self):
        r, m = ct.c_double(), ct.c_double()
        rc = lib().orc_assemble_p(self.h, ct.byref(r), ct.byref(m))
        assert rc == 0, rc
        return r.value, m.value

    def solve(self, eq):
        r0, r1 = ct.c_double(), ct.c_double()
        rc = lib().orc_solve(self.h, eq, ct.byref(r0), ct.byref(r1))
        assert rc == 0, rc
        return r0.value, r1.value

    def correct_u(self, comp):
        lib().orc_correct_u(self.h, comp)

    def correct_p(self):
        lib().orc_correct_p(self.h)

    def get(self, name):
        n = ct.c_int()
        lib().orc_case_get(self.h, name.encode(), None, ct.byref(n))
        out = np.zeros(n.value)
        rc = lib().orc_case_get(self.h, name.encode(), dp(out), ct.byref(n))
        assert rc == 0, name
        return out

    def set(self, name, arr):
        a = _d(arr).ravel()
        rc = lib().orc_case_set(self.h, name.encode(), dp(a))
        assert rc == 0, name

    def nlevels(self):
        return lib().orc_case_nlevels(self.h)

    def level(self, lvl, name):
        n = ct.c_int()
        lib().orc_level_get(self.h, lvl, name.encode(), None, ct.byref(n))
        isint = name in ("parents", "rowptr", "col", "color")
        out = np.zeros(n.value, dtype=np.int32 if isint else np.float64)
        lib().orc_level_get(self.h, lvl, name.encode(), out.ctypes.data_as(V), ct.byref(n))
        return out

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_case_destroy(self.h)
            self.h = None


# ---- stand-alone linear algebra -------------------------------------------------
def residuals(rowptr, col, ac, anb, bc, dphi):
    n = len(ac)
    r = np.zeros(n)
    lib().orc_residuals(n, ip(_i(rowptr)), ip(_i(col)), dp(_d(ac)), dp(_d(anb)), dp(_d(bc)), dp(_d(dphi)), dp(r))
    return r


def sor_sweep(rowptr, col, ac, anb, bc, dphi):
    x = _d(dphi).copy()
    lib().orc_sor_sweep(len(ac), ip(_i(rowptr)), ip(_i(col)), dp(_d(ac)), dp(_d(anb)), dp(_d(bc)), dp(x))
    return x


def ilu_factor(rowptr, col, ac, anb, quirks):
    dc = np.zeros(len(ac))
    lib().orc_ilu_factor(len(ac), ip(_i(rowptr)), ip(_i(col)), dp(_d(ac)), dp(_d(anb)), dp(dc), int(quirks))
    return dc


def ilu_sweep(rowptr, col, ac, anb, bc, dc, dphi):
    x = _d(dphi).copy()
    lib().orc_ilu_sweep(len(ac), ip(_i(rowptr)), ip(_i(col)), dp(_d(ac)), dp(_d(anb)), dp(_d(bc)), dp(_d(dc)), dp(x))
    return x


def coloring(rowptr, col):
    n = len(rowptr) - 1
    c = np.zeros(n, dtype=np.int32)
    nc = lib().orc_coloring(n, ip(_i(rowptr)), ip(_i(col)), ip(c))
    return nc, c


def mcgs_sweep(rowptr, col, ac, anb, bc, color, ncolor, dphi):
    x = _d(dphi).copy()
    lib().orc_mcgs_sweep(len(ac), ip(_i(rowptr)), ip(_i(col)), dp(_d(ac)), dp(_d(anb)), dp(_d(bc)),
                         ip(_i(color)), int(ncolor), dp(x))
    return x


def solve_algebraic_system(rowptr, col, ac, anb, bc, dphi, smoother, n_iter, rrf, quirks):
    x = _d(dphi).copy()
    r0, r1, it = ct.c_double(), ct.c_double(), ct.c_int()
    lib().orc_solve_algebraic_system(len(ac), ip(_i(rowptr)), ip(_i(col)), dp(_d(ac)), dp(_d(anb)), dp(_d(bc)),
                                     dp(x), int(smoother), int(n_iter), float(rrf), int(quirks),
                                     ct.byref(r0), ct.byref(r1), ct.byref(it))
    return x, r0.value, r1.value, it.value


def agglomerate(rowptr, col, ac, anb):
    n = len(ac)
    nnz = int(rowptr[-1])
    parents = np.zeros(n, dtype=np.int32)
    crp = np.zeros(n + 1, dtype=np.int32)
    ccol = np.zeros(nnz, dtype=np.int32)
    cac = np.zeros(n)
    canb = np.zeros(nnz)
    cn = ct.c_int()
    nc = lib().orc_agglomerate(n, ip(_i(rowptr)), ip(_i(col)), dp(_d(ac)), dp(_d(anb)), ip(parents), ip(crp),
                               ip(ccol), dp(cac), dp(canb), ct.byref(cn))
    return parents, crp[:nc + 1], ccol[:cn.value], cac[:nc], canb[:cn.value]
