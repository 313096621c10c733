"""Case descriptions for the steady SIMPLE path, in the vocabulary of uFVM's OpenFOAM inputs.

A :class:`CaseSpec` carries what uFVM reads from a case directory for this path:
``constant/polyMesh`` (mesh + physical patch types), ``0/U`` and ``0/p`` boundary
conditions, ``constant/transportProperties`` (``nu``), ``system/fvSolution``
(``nCorrectors``, ``pRefCell``, ``residualControl``, relaxation factors) and the
solver settings uFVM sets from ``run.m`` (``cfdSetupAMG`` -- ``setup/cfdSetupAMG.m:6-20``
-- and ``cfdSetupSolutionMethods`` -- ``setup/cfdSetupSolutionMethods.m:6-14``).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import meshgen
from .meshgen import PolyMesh

# physical patch types (constant/polyMesh/boundary)
PHYS = {"wall": 0, "inlet": 1, "outlet": 2, "symmetry": 3, "empty": 4}
# boundary-condition types (0/<field>)
BC = {"fixedValue": 0, "zeroGradient": 1, "noSlip": 2, "slip": 3, "empty": 4, "symmetry": 5}
SMOOTHER = {"ILU": 0, "SOR": 1, "MCGS": 2}
CYCLE = {"V-Cycle": 0, "W-Cycle": 1, "F-Cycle": 2}

# Quirk bits (set = behave like the reference; clear = repaired). Same values in the
# CUDA library (include/ufvm.h) and the oracle.
Q1_VEC_BOUNDARY_COMPONENT = 1 << 0
Q2_STRESS_NOT_TRANSPOSED = 1 << 1
Q3_NOSLIP_GAMMA_TWICE = 1 << 2
Q4_GRAD_WEIGHTS_SWAPPED = 1 << 3
Q5_ROUGH_CENTRE = 1 << 4
Q6_COARSE_DPHI_KEPT = 1 << 5
Q7_ILU_SKIP_ROW = 1 << 6
Q12_OUTLET_U_FACE_ROWS = 1 << 7
Q14_NOSLIP_PATCH_SUM = 1 << 8
Q15_NOSLIP_THIRD_SIGN = 1 << 9
Q16_ONE_CELL_COARSEST = 1 << 10
QUIRKS_REFERENCE = (1 << 11) - 1
# The reference behaviour with the three defects that stop convergence repaired: the
# patch-wide noSlip sum (Q14), which turns wall diagonals negative at low viscosity; the
# single-aggregate coarsest level (Q16), whose diagonal is ~0 for the pure-Neumann
# pressure-correction operator and divides the coarsest smoother by zero; and the coarse
# corrections kept across V-cycles (Q6), which re-adds every earlier coarse correction on each
# cycle and makes the stationary cycles of cfdApplyAMG.m diverge on fine meshes (a 234 x 234
# cavity at Re 908: the pressure-correction residual grows to 1e141 within 100 iterations).
QUIRKS_CONVERGING = QUIRKS_REFERENCE & ~(Q14_NOSLIP_PATCH_SUM | Q16_ONE_CELL_COARSEST | Q6_COARSE_DPHI_KEPT)


@dataclass
class CaseSpec:
    mesh: PolyMesh
    bc_u: List[str]                       # per patch
    bc_p: List[str]
    val_u: np.ndarray                     # (Fb, 3) boundary values (fixedValue / noSlip -> 0)
    val_p: np.ndarray                     # (Fb,)
    nu: float
    urf_u: float = 0.7
    urf_p: float = 0.3
    n_correctors: int = 2
    fixed_element: int = -1               # 0-based; -1: no reference cell
    tol_u: float = 1e-6
    tol_p: float = 1e-6
    p_amg: bool = True
    p_cycle: str = "V-Cycle"
    p_max_cycles: int = 30
    p_termination: float = 0.1
    p_max_coarse_levels: int = 10
    p_pre_sweep: int = 1
    p_post_sweep: int = 3
    p_smoother: str = "SOR"
    u_smoother: str = "ILU"
    u_n_iter: int = 10
    u_rrf: float = 0.1
    false_dt: float = 1e9
    quirks: int = QUIRKS_REFERENCE
    U0: Optional[np.ndarray] = None       # (Nc, 3)
    p0: Optional[np.ndarray] = None       # (Nc,)
    mdot0: Optional[np.ndarray] = None    # (F,)
    name: str = ""

    # flat settings shared by the oracle and the CUDA library
    def iset(self) -> np.ndarray:
        return np.array([self.n_correctors, self.fixed_element, CYCLE[self.p_cycle], self.p_max_cycles,
                         self.p_max_coarse_levels, self.p_pre_sweep, self.p_post_sweep,
                         SMOOTHER[self.p_smoother], SMOOTHER[self.u_smoother], self.u_n_iter,
                         self.quirks, int(self.p_amg)], dtype=np.int32)

    def dset(self) -> np.ndarray:
        return np.array([self.nu, self.urf_u, self.urf_p, self.tol_u, self.tol_p, self.p_termination,
                         self.u_rrf, self.false_dt], dtype=np.float64)

    def patch_types(self) -> np.ndarray:
        return np.array([PHYS[p.type] for p in self.mesh.patches], dtype=np.int32)

    def bc_codes(self):
        return (np.array([BC[t] for t in self.bc_u], dtype=np.int32),
                np.array([BC[t] for t in self.bc_p], dtype=np.int32))

    @property
    def n_cells(self) -> int:
        return self.mesh.n_cells


def _bvals(mesh: PolyMesh, u_by_patch: Dict[str, np.ndarray]):
    fb = mesh.n_faces - mesh.n_interior
    vu = np.zeros((fb, 3))
    for p in mesh.patches:
        if p.name in u_by_patch:
            vu[p.start - mesh.n_interior: p.start - mesh.n_interior + p.n] = u_by_patch[p.name]
    return vu, np.zeros(fb)


def cavity_case(n: int, nu: float = 0.01, lid: float = 1.0, dim: int = 2, nz: Optional[int] = None,
                **kw) -> CaseSpec:
    """Lid-driven cavity on the unit square/cube (lid at y = 1 moving in +x).

    ``movingWall`` fixedValue (lid 0 0), ``fixedWalls`` noSlip, ``frontAndBack`` empty (2D);
    p zeroGradient on walls with ``pRefCell 0`` (cell 0 is the reference cell).
    """
    if dim == 2:
        mesh = meshgen.cavity_hex(n, n, 1, 1.0, 1.0, 0.1)
    else:
        mesh = meshgen.cavity_hex(n, n, nz or n, 1.0, 1.0, 1.0)
    bc_u, bc_p = [], []
    for p in mesh.patches:
        if p.name == "movingWall":
            bc_u.append("fixedValue"); bc_p.append("zeroGradient")
        elif p.type == "wall":
            bc_u.append("noSlip"); bc_p.append("zeroGradient")
        else:
            bc_u.append("empty"); bc_p.append("empty")
    vu, vp = _bvals(mesh, {"movingWall": np.array([lid, 0.0, 0.0])})
    kw.setdefault("fixed_element", 0)
    kw.setdefault("name", f"cavity{dim}d_n{n}_nu{nu:g}")
    return CaseSpec(mesh=mesh, bc_u=bc_u, bc_p=bc_p, val_u=vu, val_p=vp, nu=nu, **kw)


def channel_case(nx: int = 140, ny: int = 35, nz: int = 35, nu: float = 1.0 / 200, u_max: float = 1.0,
                 jitter: float = 0.2, seed: int = 12345, **kw) -> CaseSpec:
    """Jittered 6-tet channel of a 4 x 1 x 1 box.

    Inlet (x = 0): U fixedValue u = u_max * 16 y (1 - y) z (1 - z) at face centroids
    (arithmetic mean of the triangle's nodes), p zeroGradient. Outlet (x = 4): U zeroGradient,
    p fixedValue 0. Walls: U noSlip, p zeroGradient. No reference cell.
    """
    mesh = meshgen.channel_tet(nx, ny, nz, 4.0, 1.0, 1.0, jitter, seed)
    bc_u, bc_p = [], []
    fi = mesh.n_interior
    fb = mesh.n_faces - fi
    vu = np.zeros((fb, 3)); vp = np.zeros(fb)
    for p in mesh.patches:
        if p.type == "inlet":
            bc_u.append("fixedValue"); bc_p.append("zeroGradient")
            nodes = mesh.face_nodes.reshape(-1, 3)[p.start:p.start + p.n]
            c = mesh.points[nodes].mean(axis=1)
            y, z = c[:, 1], c[:, 2]
            vu[p.start - fi:p.start - fi + p.n, 0] = u_max * 16.0 * y * (1 - y) * z * (1 - z)
        elif p.type == "outlet":
            bc_u.append("zeroGradient"); bc_p.append("fixedValue")
        else:
            bc_u.append("noSlip"); bc_p.append("zeroGradient")
    kw.setdefault("fixed_element", -1)
    kw.setdefault("name", f"channel_tet_{nx}x{ny}x{nz}")
    return CaseSpec(mesh=mesh, bc_u=bc_u, bc_p=bc_p, val_u=vu, val_p=vp, nu=nu, **kw)


def batched_sweep_params(n_cases: int = 512, seed: int = 2024, n_min: int = 16, n_max: int = 256,
                         re_min: float = 50.0, re_max: float = 1000.0):
    """Seeded (n, Re) pairs of the batched 2D-cavity sweep: n log-uniform, Re uniform."""
    rng = np.random.default_rng(seed)
    n = np.rint(np.exp(rng.uniform(np.log(n_min), np.log(n_max), size=n_cases))).astype(int)
    re = rng.uniform(re_min, re_max, size=n_cases)
    return list(zip(n.tolist(), re.tolist()))
