"""The oracle's linear-algebra pieces against direct Python transliterations of the MATLAB
loops (cfdSolveSOR.m, cfdFactorizeILU.m, cfdSolveILU.m, cfdAgglomerateLevel.m)."""
import numpy as np
import pytest

from helpers import py_agglomerate, py_ilu_factor, py_ilu_solve, py_sor, random_diag_dominant
from matlab_ufvm_b200 import case


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_sor_matches_transliteration(oracle_mod, seed):
    rp, col, ac, anb, bc = random_diag_dominant(60, seed)
    x0 = np.random.default_rng(seed).normal(size=60)
    assert np.array_equal(oracle_mod.sor_sweep(rp, col, ac, anb, bc, x0), py_sor(rp, col, ac, anb, bc, x0))


@pytest.mark.parametrize("q7", [True, False])
def test_ilu_matches_transliteration(oracle_mod, q7):
    rp, col, ac, anb, bc = random_diag_dominant(80, 3)
    q = case.QUIRKS_REFERENCE if q7 else case.QUIRKS_REFERENCE & ~case.Q7_ILU_SKIP_ROW
    dc = oracle_mod.ilu_factor(rp, col, ac, anb, q)
    assert np.array_equal(dc, py_ilu_factor(rp, col, ac, anb, q7))
    x0 = np.random.default_rng(5).normal(size=80)
    assert np.array_equal(oracle_mod.ilu_sweep(rp, col, ac, anb, bc, dc, x0), py_ilu_solve(rp, col, ac, anb, bc, dc, x0))


def _p_matrix(oracle_mod, n):
    spec = case.cavity_case(n, nu=0.01)
    oc = oracle_mod.OracleCase(spec)
    oc.update_fields()
    for c in range(3):
        oc.assemble_u(c); oc.solve(0); oc.correct_u(c)
    oc.assemble_p()
    rp = oc.mesh.get("rowptr"); col = oc.mesh.get("col")
    return rp, col, oc.get("ac"), oc.get("anb"), oc.get("bc")


@pytest.mark.parametrize("n", [6, 20])
def test_agglomeration_matches_transliteration(oracle_mod, n):
    rp, col, ac, anb, bc = _p_matrix(oracle_mod, n)
    par, crp, ccol, cac, canb = oracle_mod.agglomerate(rp, col, ac, anb)
    ppar, npar = py_agglomerate(rp, col, anb)
    assert np.array_equal(par, ppar)
    assert len(cac) == npar


def test_agglomeration_random_matrix(oracle_mod):
    rp, col, ac, anb, bc = random_diag_dominant(300, 7, nbr=6)
    par, *_ = oracle_mod.agglomerate(rp, col, ac, anb)
    ppar, _ = py_agglomerate(rp, col, anb)
    assert np.array_equal(par, ppar)


def test_coloring_is_proper_and_deterministic(oracle_mod):
    rp, col, *_ = random_diag_dominant(500, 11, nbr=6)
    nc, c1 = oracle_mod.coloring(rp, col)
    _, c2 = oracle_mod.coloring(rp, col)
    assert np.array_equal(c1, c2) and c1.min() >= 0 and c1.max() == nc - 1
    for i in range(len(rp) - 1):
        assert np.all(c1[col[rp[i]:rp[i + 1]]] != c1[i])


def _py_greedy_colouring(rp, col):
    """First-fit colouring in natural order: each row takes the smallest colour that none of
    its lower-numbered neighbours has."""
    n = len(rp) - 1
    c = np.zeros(n, dtype=np.int64)
    for i in range(n):
        used = {int(c[j]) for j in col[rp[i]:rp[i + 1]] if j < i}
        k = 0
        while k in used:
            k += 1
        c[i] = k
    return c


def _py_mcgs(rp, col, ac, anb, bc, colour, x0):
    """Symmetric multicolour Gauss-Seidel: colours ascending then descending, each row
    v = bc - sum anb * x in cconn order, x = v / ac."""
    x = np.array(x0, dtype=np.float64)
    nc = int(colour.max()) + 1
    for c in list(range(nc)) + list(range(nc - 1, -1, -1)):
        for i in np.flatnonzero(colour == c):
            v = bc[i]
            for k in range(rp[i], rp[i + 1]):
                v = v - anb[k] * x[col[k]]
            x[i] = v / ac[i]
    return x


@pytest.mark.parametrize("seed", [0, 4])
def test_mcgs_matches_transliteration(oracle_mod, seed):
    """The oracle's multicolour smoother (the multicolour form of solve/cfdSolveSOR.m:13-29)
    against the definition above: same colouring, same sweep, bit for bit."""
    rp, col, ac, anb, bc = random_diag_dominant(200, seed, nbr=6)
    nc, colour = oracle_mod.coloring(rp, col)
    assert np.array_equal(colour, _py_greedy_colouring(rp, col))
    x0 = np.random.default_rng(seed).normal(size=200)
    assert np.array_equal(oracle_mod.mcgs_sweep(rp, col, ac, anb, bc, colour, nc, x0),
                          _py_mcgs(rp, col, ac, anb, bc, colour, x0))
