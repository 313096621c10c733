"""CUDA path vs the oracle, through the C-ABI (libufvm.so). FP64 results are compared
bit for bit where the operation order is reproduced; reductions over all cells (the
residual norms) are compared at 1e-12 relative because their summation order differs."""
import numpy as np
import pytest

from helpers import cylinder_spec, random_diag_dominant, rel
from matlab_ufvm_b200 import case, meshgen

pytestmark = pytest.mark.gpu

RTOL_NORM = 1e-12


def same(a, b, name=""):
    a = np.asarray(a); b = np.asarray(b)
    assert a.shape == b.shape, (name, a.shape, b.shape)
    if not np.array_equal(a, b):
        d = np.abs(a - b)
        i = int(np.argmax(d))
        raise AssertionError(f"{name}: {np.count_nonzero(a != b)} of {a.size} differ, max |d|={d.max():.3e} "
                             f"at {i}: gpu={a.ravel()[i]!r} oracle={b.ravel()[i]!r}")


def small_channel(**kw):
    return case.channel_case(nx=8, ny=3, nz=3, **kw)


SPECS = {
    "cavity20": lambda: case.cavity_case(20, nu=0.01),
    "cavity_tutorial": lambda: case.CaseSpec(**{**case.cavity_case(20).__dict__,
                                               "mesh": meshgen.cavity_hex(20, 20, 1, 0.1, 0.1, 0.01, digits=6)}),
    "cavity3d_8": lambda: case.cavity_case(8, nu=0.0025, dim=3, p_smoother="ILU"),
    "channel_small": lambda: small_channel(),
    "cylinder": lambda: cylinder_spec()[0],
}


@pytest.mark.parametrize("name", list(SPECS))
def test_geometry_bit_exact(ufvm_mod, oracle_mod, name):
    spec = SPECS[name]()
    g = ufvm_mod.GpuCase(spec)
    om = oracle_mod.OracleMesh(spec.mesh, spec.quirks)
    for k in ("Sf", "centroid_f", "CN", "eCN", "T", "area", "gDiff", "gf", "walldist", "volume", "centroid_c"):
        same(g.geometry(k), om.get(k), k)


def _p_system(oracle_mod, spec):
    oc = oracle_mod.OracleCase(spec)
    oc.update_fields()
    for c in range(3):
        oc.assemble_u(c); oc.solve(0); oc.correct_u(c)
    oc.assemble_p()
    return oc.mesh.get("rowptr"), oc.mesh.get("col"), oc.get("ac"), oc.get("anb"), oc.get("bc")


@pytest.mark.parametrize("which", ["random", "cavity"])
def test_residual_sor_ilu_bit_exact(ufvm_mod, oracle_mod, which):
    if which == "random":
        rp, col, ac, anb, bc = random_diag_dominant(3000, 1, nbr=6)
    else:
        rp, col, ac, anb, bc = _p_system(oracle_mod, case.cavity_case(32, nu=0.01))
    x0 = np.random.default_rng(2).normal(size=len(ac)) * 1e-3
    same(ufvm_mod.cfdComputeResidualsArray(rp, col, ac, anb, bc, x0), oracle_mod.residuals(rp, col, ac, anb, bc, x0),
         "residual")
    same(ufvm_mod.cfdSolveSOR(rp, col, ac, anb, bc, x0), oracle_mod.sor_sweep(rp, col, ac, anb, bc, x0), "SOR")
    for q in (case.QUIRKS_REFERENCE, 0):
        dc = ufvm_mod.cfdFactorizeILU(rp, col, ac, anb, q)
        same(dc, oracle_mod.ilu_factor(rp, col, ac, anb, q), "ILU factor")
    same(ufvm_mod.cfdSolveILU(rp, col, ac, anb, bc, dc, x0), oracle_mod.ilu_sweep(rp, col, ac, anb, bc, dc, x0),
         "ILU solve")
    for sm in ("ILU", "SOR", "MCGS"):
        xg, r0g, r1g, itg = ufvm_mod.cfdSolveAlgebraicSystem(rp, col, ac, anb, bc, x0, sm, 10, 0.1)
        xo, r0o, r1o, ito = oracle_mod.solve_algebraic_system(rp, col, ac, anb, bc, x0, case.SMOOTHER[sm], 10, 0.1,
                                                              case.QUIRKS_REFERENCE)
        assert itg == ito, sm
        same(xg, xo, "cfdSolveAlgebraicSystem " + sm)
        assert abs(r0g - r0o) <= RTOL_NORM * abs(r0o) and abs(r1g - r1o) <= RTOL_NORM * abs(r1o)


@pytest.mark.parametrize("which", ["random", "cavity"])
def test_profiled_kernels_do_the_work(ufvm_mod, oracle_mod, which):
    """The kernel-timing entry point times the real sweeps: after it, dphi equals 1 + reps
    sweeps of the oracle (one untimed launch, then reps timed ones), bit for bit."""
    import torch
    if which == "random":
        rp, col, ac, anb, bc = random_diag_dominant(3000, 5, nbr=6)
    else:
        rp, col, ac, anb, bc = _p_system(oracle_mod, case.cavity_case(24, nu=0.01))
    x0 = np.random.default_rng(3).normal(size=len(ac)) * 1e-3
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (rp, col, ac, anb, bc)]
    reps = 2
    nc, color = oracle_mod.coloring(rp, col)
    dc = oracle_mod.ilu_factor(rp, col, ac, anb, 0)
    step = {"SOR": lambda x: oracle_mod.sor_sweep(rp, col, ac, anb, bc, x),
            "MCGS": lambda x: oracle_mod.mcgs_sweep(rp, col, ac, anb, bc, color, nc, x),
            "ILU": lambda x: oracle_mod.ilu_sweep(rp, col, ac, anb, bc, dc, x)}
    for name, f in step.items():
        x = torch.from_numpy(x0.copy()).cuda()
        ms, by = ufvm_mod.profile_plain_kernel(name, *dev, x, reps)
        assert ms > 0 and by > 0
        want = x0.copy()
        for _ in range(1 + reps):
            want = f(want)
        same(x.cpu().numpy(), want, "profiled " + name)
    x = torch.from_numpy(x0.copy()).cuda()
    ms, by = ufvm_mod.profile_plain_kernel("residual", *dev, x, reps)
    assert ms > 0 and by == 36.0 * len(ac) + 12.0 * len(col)
    same(x.cpu().numpy(), x0, "residual leaves dphi")


@pytest.mark.parametrize("which", ["random", "cavity20", "cavity64", "channel"])
def test_agglomeration_bit_exact(ufvm_mod, oracle_mod, which):
    if which == "random":
        rp, col, ac, anb, bc = random_diag_dominant(5000, 4, nbr=6)
    elif which == "channel":
        rp, col, ac, anb, bc = _p_system(oracle_mod, small_channel())
    else:
        rp, col, ac, anb, bc = _p_system(oracle_mod, case.cavity_case(int(which[6:]), nu=0.01))
    g = ufvm_mod.cfdAgglomerateLevel(rp, col, ac, anb)
    o = oracle_mod.agglomerate(rp, col, ac, anb)
    for a, b, n in zip(g, o, ("parents", "coarse rowptr", "coarse col", "coarse ac", "coarse anb")):
        same(a, b, n)


FIELDS_CELL = ("U", "p", "gradU", "gradp", "DU", "PP", "gradPP")


def _compare_case(g, oc, names=FIELDS_CELL + ("mdot", "fluxC1", "fluxC2", "ac", "bc", "anb", "dphi")):
    for n in names:
        same(g.get(n), oc.get(n), n)


@pytest.mark.parametrize("name", ["cavity20", "cavity3d_8", "channel_small", "cylinder"])
def test_stage_by_stage_bit_exact(ufvm_mod, oracle_mod, name):
    spec = SPECS[name]()
    g = ufvm_mod.GpuCase(spec)
    oc = oracle_mod.OracleCase(spec)
    _compare_case(g, oc, ("U", "p", "gradU", "gradp", "mdot"))
    for it in range(2):
        g.cfdUpdateFields(); oc.update_fields()
        assert g.get("scaleU")[0] == oc.get("scaleU")[0]
        _compare_case(g, oc, ("U", "p", "gradU", "gradp"))
        for c in range(3):
            rg = g.cfdAssembleEquation("U", c + 1)
            ro = oc.assemble_u(c)
            _compare_case(g, oc, ("ac", "bc", "anb", "DU"))
            assert rel(rg, ro) < RTOL_NORM
            sg = g.cfdSolveEquation("U"); so = oc.solve(0)
            same(g.get("dphi"), oc.get("dphi"), f"U{c} dphi it{it}")
            assert rel(sg, so) < RTOL_NORM
            g.cfdCorrectEquation("U", c + 1); oc.correct_u(c)
            same(g.get("U"), oc.get("U"), f"U after correct {c}")
        for k in range(spec.n_correctors):
            rg = g.cfdAssembleEquation("p"); ro = oc.assemble_p()
            _compare_case(g, oc, ("mdot", "fluxC1", "fluxC2", "ac", "bc", "anb"))
            assert rel(rg, ro) < RTOL_NORM
            sg = g.cfdSolveEquation("p"); so = oc.solve(1)
            assert g.levels() == [len(oc.level(l, "ac")) for l in range(oc.nlevels())]
            for l in range(oc.nlevels() - 1):
                same(g.level_array(l, "parents"), oc.level(l, "parents"), f"parents level {l}")
            same(g.get("dphi"), oc.get("dphi"), f"p dphi it{it} corr{k}")
            assert rel(sg, so) < RTOL_NORM
            g.cfdCorrectEquation("p"); oc.correct_p()
            _compare_case(g, oc, ("U", "p", "PP", "gradPP", "mdot"))


@pytest.mark.parametrize("name,iters", [("cavity20", 10), ("channel_small", 4), ("cylinder", 5),
                                        ("cavity20_mcgs", 6), ("cavity32_fcycle", 6), ("cavity32_fcycle_sor", 6)])
def test_iterations_bit_exact(ufvm_mod, oracle_mod, name, iters):
    if name == "cavity20_mcgs":  # the multicolour smoother for U and p inside the AMG
        spec = case.CaseSpec(**{**case.cavity_case(20, nu=0.01).__dict__, "p_smoother": "MCGS", "u_smoother": "MCGS"})
    elif name.startswith("cavity32_fcycle"):
        # the F-cycle of solve/AMG/cfdApplyFCycle.m for p (ILU or Gauss-Seidel smoothing)
        spec = case.cavity_case(32, nu=0.005, p_cycle="F-Cycle", p_smoother="SOR" if name.endswith("sor") else "ILU")
    else:
        spec = SPECS[name]()
    g = ufvm_mod.GpuCase(spec)
    oc = oracle_mod.OracleCase(spec)
    for it in range(iters):
        rg, cg = g.iterate()
        rc, ro = oc.iterate()
        assert np.allclose(rg, ro, rtol=1e-10, atol=0), (it, rg, ro)
    _compare_case(g, oc, ("U", "p", "mdot"))


def test_cylinder_kat_on_gpu(ufvm_mod):
    spec, z = cylinder_spec()
    g = ufvm_mod.GpuCase(spec)
    for _ in range(5):
        g.iterate()
    nc, fi = spec.mesh.n_cells, spec.mesh.n_interior
    U = g.get("U").reshape(3, -1)[:, :nc].T
    assert rel(U, z["U_045"]) < 1e-5 and rel(g.get("p")[:nc], z["p_045"]) < 1e-5
    assert rel(g.get("mdot")[:fi], z["mdot_045"][:fi]) < 1e-5


def test_c1_cavity_converges_like_oracle(ufvm_mod, oracle_mod):
    spec = case.cavity_case(20, nu=0.01)
    g = ufvm_mod.GpuCase(spec)
    itg, rg = g.cfdRunCase(500)
    oc = oracle_mod.OracleCase(spec)
    for ito in range(1, 501):
        rc, ro = oc.iterate()
        if rc != 0:
            break
    assert itg == ito == 58
    assert rel(g.get("U"), oc.get("U")) < 1e-12 and rel(g.get("p"), oc.get("p")) < 1e-12


# The named workloads at full size: the 64^3 cavity (262,144 cells, ILU for p) and the
# 1,029,000-cell jittered-tet channel, against the oracle bit for bit. Large working sets (the
# 64^3 pressure system and the channel's geometry exceed the L2 of a B200 together with the
# fields) exercise the level schedules with hundreds of levels and the block grids at scale.
FULL = {
    "cavity3d_64_ilu": (lambda: case.cavity_case(64, nu=1.0 / 400, dim=3, p_smoother="ILU"), 2),
    "channel_1M_tet": (lambda: case.channel_case(), 1),
}


@pytest.mark.parametrize("name", list(FULL))
def test_full_size_configs_bit_exact(ufvm_mod, oracle_mod, name):
    make, iters = FULL[name]
    spec = make()
    g = ufvm_mod.GpuCase(spec)
    oc = oracle_mod.OracleCase(spec)
    om = oracle_mod.OracleMesh(spec.mesh, spec.quirks)
    for k in ("volume", "gDiff", "gf", "Sf"):
        same(g.geometry(k), om.get(k), k)
    vol = g.geometry("volume")
    assert abs(vol.sum() - (4.0 if "channel" in name else 1.0)) < 1e-9
    for it in range(iters):
        rg, _ = g.iterate()
        _, ro = oc.iterate()
        assert np.all(np.isfinite(rg[:4]))
        assert np.allclose(rg[:8], ro[:8], rtol=1e-10, atol=0), (it, rg[:8], ro[:8])
    _compare_case(g, oc, ("U", "p", "mdot"))
    g.close()


def test_gpu_restart_from_checkpoint_bit_exact(ufvm_mod, tmp_path):
    """A GPU case checkpointed to OpenFOAM fields and restarted continues bit for bit."""
    import dataclasses
    from matlab_ufvm_b200 import polymesh
    spec = case.cavity_case(16, nu=0.01)
    straight = ufvm_mod.GpuCase(spec)
    for _ in range(5):
        straight.iterate()
    first = ufvm_mod.GpuCase(spec)
    for _ in range(3):
        first.iterate()
    polymesh.write_time_directory(str(tmp_path), "3", spec, first.get("U"), first.get("p"), first.get("mdot"))
    U0, p0, m0 = polymesh.read_time_directory(str(tmp_path), "3", spec.mesh)
    resumed = ufvm_mod.GpuCase(dataclasses.replace(spec, U0=U0, p0=p0, mdot0=m0))
    for _ in range(2):
        resumed.iterate()
    for name in ("U", "p", "mdot"):
        same(straight.get(name), resumed.get(name), name)
