"""Shared test helpers: fixture loading and small pure-Python restatements."""
import os

import numpy as np

from matlab_ufvm_b200 import case, meshgen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def cylinder_spec(quirks=case.QUIRKS_REFERENCE, **kw):
    z = np.load(os.path.join(GOLDEN, "cylinder_kat.npz"))
    mesh = meshgen.PolyMesh(points=z["points"], face_start=z["face_start"], face_nodes=z["face_nodes"],
                            owner=z["owner"], neighbour=z["neighbour"],
                            patches=[meshgen.Patch(str(n), str(t), int(s), int(c)) for n, t, s, c in
                                     zip(z["patch_names"], z["patch_types"], z["patch_start"], z["patch_n"])])
    fb = mesh.n_faces - mesh.n_interior
    args = dict(p_cycle="W-Cycle", n_correctors=2, fixed_element=-1, p_smoother="ILU", u_smoother="ILU",
                U0=z["U_04"], p0=z["p_04"], mdot0=z["mdot_04"])
    args.update(kw)
    spec = case.CaseSpec(mesh=mesh, bc_u=[str(x) for x in z["bc_u"]], bc_p=[str(x) for x in z["bc_p"]],
                         val_u=z["val_u"], val_p=np.zeros(fb), nu=float(z["nu"]), quirks=quirks, **args)
    return spec, z


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def random_diag_dominant(n, seed=0, nbr=4):
    """Random symmetric-pattern matrix in cconn-ordered CSR (rows list neighbours)."""
    rng = np.random.default_rng(seed)
    adj = [set() for _ in range(n)]
    for i in range(n):
        for _ in range(nbr // 2):
            j = int(rng.integers(0, n))
            if j != i:
                adj[i].add(j); adj[j].add(i)
    rowptr = [0]
    col = []
    for i in range(n):
        nb = sorted(adj[i], key=lambda j: (rng.random(), j))
        col += nb
        rowptr.append(len(col))
    rowptr = np.array(rowptr, dtype=np.int32)
    col = np.array(col, dtype=np.int32)
    anb = -rng.uniform(0.1, 1.0, size=len(col))
    ac = np.array([-anb[rowptr[i]:rowptr[i + 1]].sum() * rng.uniform(1.05, 1.5) + 1e-3 for i in range(n)])
    bc = rng.normal(size=n)
    return rowptr, col, ac, anb, bc


# ---- direct transliterations of the MATLAB smoothers (1-based loops kept as written)
def py_sor(rowptr, col, ac, anb, bc, dphi):
    x = np.array(dphi, dtype=np.float64)
    n = len(ac)
    for i in list(range(n)) + list(range(n - 1, -1, -1)):
        v = bc[i]
        for k in range(rowptr[i], rowptr[i + 1]):
            v = v - anb[k] * x[col[k]]
        x[i] = v / ac[i]
    return x


def py_ilu_factor(rowptr, col, ac, anb, q7=True):
    n = len(ac)
    dc = np.array(ac, dtype=np.float64)
    for i1 in range(1, n + 1):
        dc[i1 - 1] = 1.0 / dc[i1 - 1]
        if (i1 != n - 1) or not q7:
            for j1_ in range(rowptr[i1 - 1], rowptr[i1]):
                jj1 = col[j1_] + 1
                if jj1 > i1:
                    for i1_ in range(rowptr[jj1 - 1], rowptr[jj1]):
                        if col[i1_] + 1 == i1:
                            break
                    dc[jj1 - 1] = dc[jj1 - 1] - anb[i1_] * dc[i1 - 1] * anb[j1_]
    return dc


def py_ilu_solve(rowptr, col, ac, anb, bc, dc, dphi):
    n = len(ac)
    x = np.array(dphi, dtype=np.float64)
    rc = np.zeros(n)
    for i in range(n):
        res = -ac[i] * x[i] + bc[i]
        for k in range(rowptr[i], rowptr[i + 1]):
            res = res - anb[k] * x[col[k]]
        rc[i] = res
    for i1 in range(n):
        mat1 = dc[i1] * rc[i1]
        for k in range(rowptr[i1], rowptr[i1 + 1]):
            j1 = col[k]
            if j1 > i1:
                for q in range(rowptr[j1], rowptr[j1 + 1]):
                    if col[q] == i1:
                        break
                rc[j1] = rc[j1] - anb[q] * mat1
    for i1 in range(n - 1, -1, -1):
        if i1 < n - 1:
            for k in range(rowptr[i1], rowptr[i1 + 1]):
                j = col[k]
                if j > i1:
                    rc[i1] = rc[i1] - anb[k] * rc[j]
        mat1 = dc[i1] * rc[i1]
        rc[i1] = mat1
        x[i1] = x[i1] + mat1
    return x


def py_agglomerate(rowptr, col, anb):
    n = len(rowptr) - 1
    parents = np.zeros(n, dtype=np.int64)
    maxAnb = np.array([max(-anb[rowptr[i]:rowptr[i + 1]]) for i in range(n)])
    iParent = 1
    for s in range(n):
        if parents[s] == 0:
            parents[s] = iParent
            children = [s]
            for k in range(rowptr[s], rowptr[s + 1]):
                nb = col[k]
                if parents[nb] == 0 and (-anb[k] / maxAnb[s]) > 0.5:
                    parents[nb] = iParent
                    children.append(nb)
            children2 = []
            for c in children[1:]:
                for k in range(rowptr[c], rowptr[c + 1]):
                    nb = col[k]
                    if parents[nb] == 0 and (-anb[k] / maxAnb[c]) > 0.5:
                        parents[nb] = iParent
                        children2.append(nb)
            if len(children) + len(children2) == 1:
                parents[s] = 0
            else:
                iParent += 1
    for o in range(n):
        if parents[o] == 0:
            strength = 0.0
            for k in range(rowptr[o], rowptr[o + 1]):
                nb = col[k]
                if parents[nb] != 0 and strength < -anb[k] / maxAnb[nb]:
                    strength = -anb[k] / maxAnb[nb]
                    parents[o] = parents[nb]
        if parents[o] == 0:
            parents[o] = iParent
            iParent += 1
    return (parents - 1).astype(np.int32), iParent - 1
