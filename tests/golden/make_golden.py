"""Generates the golden fixtures in this directory from the reference's own data files.

Run where a checkout of the reference exists, with UFVM_REFERENCE set to its ``uFVM`` directory
(the one holding ``src/`` and ``tutorials/``); the script refuses to run without it. It reads
only data the reference ships:

* ``tutorials/basic/cavity1/constant/polyMesh/theMesh.mat`` -- the fully processed mesh
  struct written by uFVM itself (utilities/extras/cfdGenerateInitialResults.m:16-23):
  the geometry known-answer test for cfdProcessOpenFoamMesh;
* ``tutorials/basic/cavity1/constant/polyMesh/{points,faces,owner,neighbour,boundary}``:
  hashes of the raw polyMesh, to pin the cavity generator;
* ``tutorials/incompressible/cylinder/{constant/polyMesh, 0.4, 0.45}``: the steady SIMPLE
  snapshots uFVM wrote every 5 iterations (cfdWriteOpenFoamField.m:21-80, ~5 significant
  digits): the integration known-answer test (restart from 0.4, 5 iterations, compare 0.45).

Outputs: ``cavity1_theMesh.npz``, ``cavity1_polymesh_sha256.json``, ``cylinder_kat.npz``.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from matlab_ufvm_b200 import polymesh  # noqa: E402

REF = os.environ.get("UFVM_REFERENCE", "")


def the_mesh():
    import scipy.io as sio
    mat = sio.loadmat(os.path.join(REF, "tutorials/basic/cavity1/constant/polyMesh/theMesh.mat"),
                      squeeze_me=False, struct_as_record=False)["theMesh"][0, 0]
    faces = mat.faces[0]
    els = mat.elements[0]
    fi = int(mat.numberOfInteriorFaces[0, 0])

    def fvec(n):
        return np.array([getattr(f, n).ravel() for f in faces], dtype=np.float64)

    def fsc(n):
        return np.array([getattr(f, n).ravel()[0] for f in faces], dtype=np.float64)

    out = dict(
        Sf=fvec("Sf"), centroid_f=fvec("centroid"), CN=fvec("CN"), eCN=fvec("eCN"), T=fvec("T"),
        area=fsc("area"), gDiff=fsc("gDiff"), gf=fsc("gf"), walldist=fsc("walldist"),
        volume=np.array([e.volume.ravel()[0] for e in els]),
        centroid_c=np.array([e.centroid.ravel() for e in els]),
        own_coef=np.array([faces[f].iOwnerNeighbourCoef.ravel()[0] for f in range(fi)], dtype=np.int32) - 1,
        nei_coef=np.array([faces[f].iNeighbourOwnerCoef.ravel()[0] for f in range(fi)], dtype=np.int32) - 1,
    )
    cc = [np.atleast_1d(c[0].ravel()).astype(np.int32) - 1 for c in mat.cconn]
    out["cconn_rowptr"] = np.concatenate([[0], np.cumsum([len(c) for c in cc])]).astype(np.int32)
    out["cconn_col"] = np.concatenate(cc).astype(np.int32)
    np.savez_compressed(os.path.join(HERE, "cavity1_theMesh.npz"), **out)


def polymesh_hashes():
    m = polymesh.read_polymesh(os.path.join(REF, "tutorials/basic/cavity1"))
    h = {k: hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest()
         for k, v in (("points", m.points), ("face_start", m.face_start.astype(np.int32)),
                      ("face_nodes", m.face_nodes.astype(np.int32)), ("owner", m.owner.astype(np.int32)),
                      ("neighbour", m.neighbour.astype(np.int32)))}
    h["patches"] = [[p.name, p.type, p.start, p.n] for p in m.patches]
    with open(os.path.join(HERE, "cavity1_polymesh_sha256.json"), "w") as f:
        json.dump(h, f, indent=1)


def cylinder():
    case = os.path.join(REF, "tutorials/incompressible/cylinder")
    m = polymesh.read_polymesh(case)
    out = dict(points=m.points, face_start=m.face_start, face_nodes=m.face_nodes, owner=m.owner,
               neighbour=m.neighbour, patch_start=np.array([p.start for p in m.patches], np.int32),
               patch_n=np.array([p.n for p in m.patches], np.int32))
    names = [p.name for p in m.patches]
    types = [p.type for p in m.patches]
    fi = m.n_interior
    nb = m.n_faces - fi
    for t in ("0.4", "0.45"):
        tag = t.replace(".", "")
        U = polymesh.read_field(os.path.join(case, t, "U"))
        p = polymesh.read_field(os.path.join(case, t, "p"))
        md = polymesh.read_field(os.path.join(case, t, "mdot_f"))
        out[f"U_{tag}"] = U["internal"][1]
        out[f"p_{tag}"] = p["internal"][1]
        mdot = np.zeros(m.n_faces)
        mdot[:fi] = md["internal"][1]
        for pch in m.patches:
            v = md["boundary"][pch.name]["value"]
            mdot[pch.start:pch.start + pch.n] = v[1]
        out[f"mdot_{tag}"] = mdot
    U0 = polymesh.read_field(os.path.join(case, "0", "U"))
    p0 = polymesh.read_field(os.path.join(case, "0", "p"))
    out["bc_u"] = np.array([U0["boundary"][n]["type"] for n in names])
    out["bc_p"] = np.array([p0["boundary"][n]["type"] for n in names])
    out["patch_names"] = np.array(names)
    out["patch_types"] = np.array(types)
    vu = np.zeros((nb, 3))
    for pch in m.patches:
        ent = U0["boundary"][pch.name]
        if "value" in ent:
            vu[pch.start - fi:pch.start - fi + pch.n] = ent["value"][1]
    out["val_u"] = vu
    out["nu"] = np.array(1.4775e-5)
    np.savez_compressed(os.path.join(HERE, "cylinder_kat.npz"), **out)


if __name__ == "__main__":
    if not REF or not os.path.isdir(os.path.join(REF, "tutorials")):
        sys.exit("set UFVM_REFERENCE to the reference's uFVM directory (the one holding src/ and tutorials/)")
    the_mesh()
    polymesh_hashes()
    cylinder()
    print("fixtures written to", HERE)
