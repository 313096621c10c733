"""OpenFOAM ASCII readers/writers for polyMesh directories and volume/surface fields.

Reads the same files uFVM's ``src/utilities/IO/cfdReadPolyMesh.m:17-214`` reads
(``points``, ``faces``, ``owner``, ``neighbour``, ``boundary``) and the time-directory
fields ``cfdReadTimeDirectory.m`` reads (``internalField`` uniform / nonuniform,
per-patch ``boundaryField`` with ``type`` and ``value``).  Indices stay 0-based.
"""
from __future__ import annotations

import os
import re
from typing import Dict, List, Tuple

import numpy as np

from .meshgen import Patch, PolyMesh

_COMMENT = re.compile(r"//[^\n]*|/\*.*?\*/", re.S)


def _strip(text: str) -> str:
    return _COMMENT.sub(" ", text)


def _body_after_header(text: str) -> str:
    text = _strip(text)
    m = re.search(r"FoamFile\s*\{.*?\}", text, re.S)
    return text[m.end():] if m else text


def _read_list_block(text: str) -> Tuple[int, str]:
    """Return (count, inside-of-outer-parentheses) for the first ``N ( ... )`` list."""
    m = re.search(r"(\d+)\s*\(", text)
    n = int(m.group(1))
    depth = 0
    start = m.end() - 1
    for pos in range(start, len(text)):
        ch = text[pos]
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
            if depth == 0:
                return n, text[start + 1:pos]
    raise ValueError("unterminated list")


def read_points(path: str) -> np.ndarray:
    n, body = _read_list_block(_body_after_header(open(path).read()))
    vals = np.array(body.replace("(", " ").replace(")", " ").split(), dtype=np.float64)
    return vals.reshape(n, 3)


def read_faces(path: str) -> Tuple[np.ndarray, np.ndarray]:
    n, body = _read_list_block(_body_after_header(open(path).read()))
    toks = body.replace("(", " ( ").replace(")", " ) ").split()
    start = [0]
    nodes: List[int] = []
    it = iter(toks)
    for tok in it:
        if tok == "(" or tok == ")":
            continue
        cnt = int(tok)
        assert next(it) == "("
        for _ in range(cnt):
            nodes.append(int(next(it)))
        assert next(it) == ")"
        start.append(len(nodes))
    assert len(start) == n + 1
    return np.asarray(start, dtype=np.int32), np.asarray(nodes, dtype=np.int32)


def read_label_list(path: str) -> np.ndarray:
    n, body = _read_list_block(_body_after_header(open(path).read()))
    return np.asarray(body.split(), dtype=np.int32)[:n]


def read_boundary(path: str) -> List[Patch]:
    body = _body_after_header(open(path).read())
    n, inner = _read_list_block(body)
    patches = []
    for m in re.finditer(r"(\w+)\s*\{(.*?)\}", inner, re.S):
        name, blk = m.group(1), m.group(2)
        ptype = re.search(r"\btype\s+(\w+)\s*;", blk).group(1)
        nf = int(re.search(r"\bnFaces\s+(\d+)\s*;", blk).group(1))
        sf = int(re.search(r"\bstartFace\s+(\d+)\s*;", blk).group(1))
        patches.append(Patch(name, ptype, sf, nf))
    assert len(patches) == n
    return patches


def read_polymesh(case_dir: str) -> PolyMesh:
    d = os.path.join(case_dir, "constant", "polyMesh")
    pts = read_points(os.path.join(d, "points"))
    fs, fn = read_faces(os.path.join(d, "faces"))
    own = read_label_list(os.path.join(d, "owner"))
    nei = read_label_list(os.path.join(d, "neighbour"))
    patches = read_boundary(os.path.join(d, "boundary"))
    return PolyMesh(points=pts, face_start=fs, face_nodes=fn, owner=own, neighbour=nei, patches=patches)


def _parse_value(txt: str, ncomp: int):
    txt = txt.strip()
    if txt.startswith("uniform"):
        rest = txt[len("uniform"):].replace("(", " ").replace(")", " ").split()
        v = np.array(rest, dtype=np.float64)
        return ("uniform", v if ncomp > 1 else float(v[0]))
    if txt.startswith("nonuniform"):
        n, body = _read_list_block(txt)
        v = np.array(body.replace("(", " ").replace(")", " ").split(), dtype=np.float64)
        return ("nonuniform", v.reshape(n, ncomp) if ncomp > 1 else v)
    raise ValueError(txt[:40])


def read_field(path: str) -> Dict:
    """Read a vol/surface field: ``{'class', 'internal': (kind, value), 'boundary': {patch: {...}}}``."""
    raw = _strip(open(path).read())
    cls = re.search(r"\bclass\s+(\w+)\s*;", raw).group(1)
    ncomp = 3 if "Vector" in cls else 1
    body = _body_after_header(raw)
    m = re.search(r"internalField\s+(.*?);\s*boundaryField", body, re.S)
    internal = _parse_value(m.group(1), ncomp)
    bstart = body.index("boundaryField")
    bbody = body[body.index("{", bstart) + 1:]
    boundary = {}
    pos = 0
    while True:
        m = re.compile(r"(\w+)\s*\{").search(bbody, pos)
        if not m:
            break
        name = m.group(1)
        depth = 0
        for q in range(m.end() - 1, len(bbody)):
            if bbody[q] == "{":
                depth += 1
            elif bbody[q] == "}":
                depth -= 1
                if depth == 0:
                    break
        blk = bbody[m.end():q]
        ent = {"type": re.search(r"\btype\s+(\w+)\s*;", blk).group(1)}
        vm = re.search(r"\bvalue\s+(.*?);", blk, re.S)
        if vm:
            ent["value"] = _parse_value(vm.group(1), ncomp)
        boundary[name] = ent
        pos = q + 1
    return {"class": cls, "ncomp": ncomp, "internal": internal, "boundary": boundary}


def write_polymesh(mesh: PolyMesh, case_dir: str) -> None:
    """Write an ASCII polyMesh that ``cfdReadPolyMesh`` can read (18-line headers)."""
    d = os.path.join(case_dir, "constant", "polyMesh")
    os.makedirs(d, exist_ok=True)

    def header(cls, obj):
        return ("/*--------------------------------*- C++ -*----------------------------------*\\\n"
                "  generated by matlab_ufvm_b200.polymesh\n"
                "\\*---------------------------------------------------------------------------*/\n"
                "FoamFile\n{\n    version     2.0;\n    format      ascii;\n"
                f"    class       {cls};\n    location    \"constant/polyMesh\";\n    object      {obj};\n}}\n"
                "// * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * //\n\n\n")
    with open(os.path.join(d, "points"), "w") as f:
        f.write(header("vectorField", "points"))
        f.write(f"{mesh.points.shape[0]}\n(\n")
        for p in mesh.points:
            f.write(f"({p[0]:.17g} {p[1]:.17g} {p[2]:.17g})\n")
        f.write(")\n")
    with open(os.path.join(d, "faces"), "w") as f:
        f.write(header("faceList", "faces"))
        nf = mesh.n_faces
        f.write(f"{nf}\n(\n")
        for i in range(nf):
            nodes = mesh.face_nodes[mesh.face_start[i]:mesh.face_start[i + 1]]
            f.write(f"{len(nodes)}(" + " ".join(str(int(x)) for x in nodes) + ")\n")
        f.write(")\n")
    for name, arr in (("owner", mesh.owner), ("neighbour", mesh.neighbour)):
        with open(os.path.join(d, name), "w") as f:
            f.write(header("labelList", name))
            f.write(f"{arr.shape[0]}\n(\n" + "\n".join(str(int(x)) for x in arr) + "\n)\n")
    with open(os.path.join(d, "boundary"), "w") as f:
        f.write(header("polyBoundaryMesh", "boundary")[:-1])
        f.write(f"{len(mesh.patches)}\n(\n")
        for p in mesh.patches:
            f.write(f"    {p.name}\n    {{\n        type            {p.type};\n"
                    f"        nFaces          {p.n};\n        startFace       {p.start};\n    }}\n")
        f.write(")\n")


_BS = chr(92) * 2  # the reference's banner lines carry two backslashes
_FOAM_BANNER = "\n".join([
    "/*--------------------------------*- C++ -*----------------------------------*" + _BS,
    "| =========                 |                                                 |",
    "| " + _BS + "      /  F ield         | OpenFOAM: The Open Source CFD Toolbox           |",
    "|  " + _BS + "    /   O peration     | Version:  v1706                                 |",
    "|   " + _BS + "  /    A nd           | Web:      www.OpenFOAM.com                      |",
    "|    " + _BS + "/     M anipulation  |                                                 |",
    _BS + "*---------------------------------------------------------------------------*/",
]) + "\n"

_DIMENSIONS = {"U": "[0 1 -1 0 0 0 0]", "p": "[0 2 -2 0 0 0 0]", "mdot_f": "[1 0 -1 0 0 0 0]"}


def _fmt(x: float, digits: int) -> str:
    return f"{x:.{digits}g}"


def _value_block(values: np.ndarray, ncomp: int, digits: int, indent: str) -> List[str]:
    kind = "vector" if ncomp == 3 else "scalar"
    out = [f"{indent}nonuniform List<{kind}>", str(len(values)), "("]
    if ncomp == 3:
        out += ["(" + " ".join(_fmt(v, digits) for v in row) + ")" for row in np.asarray(values).reshape(-1, 3)]
    else:
        out += [_fmt(v, digits) for v in np.asarray(values).ravel()]
    return out + [")", ";"]


def write_field(path: str, name: str, cls: str, internal: np.ndarray, boundary: List[Tuple[str, str, object]],
                location: str = "0", dimensions: str = None, digits: int = 17) -> None:
    """Write a field in the layout of postProcess/cfdWriteOpenFoamField.m (header, dimensions,
    ``internalField nonuniform List<...>``, then per patch ``type`` and an optional nonuniform
    ``value``). ``boundary`` lists (patch name, type, values or None) in patch order.
    ``digits`` 17 writes every double exactly (a restart continues bit for bit); the reference
    prints 5 significant digits (MATLAB num2str), which ``digits=5`` reproduces."""
    ncomp = 3 if "Vector" in cls else 1
    lines = [_FOAM_BANNER.rstrip("\n"), "FoamFile", "{", "    version     2.0;", "    format      ascii;",
             f"    class       {cls};", f'    location    "{location}";', f"    object      {name};", "}",
             "// * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * //", "",
             f"dimensions      {dimensions or _DIMENSIONS.get(name, '[0 0 0 0 0 0 0]')}", "", ""]
    body = _value_block(internal, ncomp, digits, "internalField   ")
    lines += body
    lines += ["", "boundaryField", "{"]
    for pname, ptype, vals in boundary:
        lines += [f"    {pname}", "    {", f"        type             {ptype};"]
        if vals is not None:
            lines += _value_block(vals, ncomp, digits, "        value            ")
        lines += ["    }"]
    lines += ["}", ""]
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write("\n".join(lines))


def write_time_directory(case_dir: str, time: str, spec, U: np.ndarray, p: np.ndarray, mdot: np.ndarray,
                         digits: int = 17) -> str:
    """Checkpoint a steady state: U, p and mdot_f of a case (rows as the C-ABI returns them:
    U as 3 x (cells + boundary faces), p as cells + boundary faces, mdot per face) into
    ``case_dir/time`` in OpenFOAM format. Returns the directory."""
    m = spec.mesh
    nc, fi = m.n_cells, m.n_interior
    d = os.path.join(case_dir, time)
    U = np.asarray(U, dtype=np.float64).reshape(3, -1)
    p = np.asarray(p, dtype=np.float64).ravel()
    mdot = np.asarray(mdot, dtype=np.float64).ravel()
    ub, pb, fb = [], [], []
    for patch, tu, tp in zip(m.patches, spec.bc_u, spec.bc_p):
        lo, hi = nc + patch.start - fi, nc + patch.start - fi + patch.n
        ub.append((patch.name, tu, None if tu == "empty" else U[:, lo:hi].T))
        pb.append((patch.name, tp, None if tp == "empty" else p[lo:hi]))
        fb.append((patch.name, "calculated", None if tp == "empty" else mdot[patch.start:patch.start + patch.n]))
    write_field(os.path.join(d, "U"), "U", "volVectorField", U[:, :nc].T, ub, time, digits=digits)
    write_field(os.path.join(d, "p"), "p", "volScalarField", p[:nc], pb, time, digits=digits)
    write_field(os.path.join(d, "mdot_f"), "mdot_f", "surfaceScalarField", mdot[:fi], fb, time, digits=digits)
    return d


def read_time_directory(case_dir: str, time: str, mesh: PolyMesh):
    """The (U0, p0, mdot0) initial fields of a restart from ``case_dir/time``:
    U0 (cells, 3), p0 (cells,), mdot0 (faces,) with the boundary faces' mdot from the patches."""
    d = os.path.join(case_dir, time)
    fu, fp, fm = read_field(os.path.join(d, "U")), read_field(os.path.join(d, "p")), read_field(os.path.join(d, "mdot_f"))
    U0 = np.asarray(fu["internal"][1], dtype=np.float64).reshape(-1, 3)
    p0 = np.asarray(fp["internal"][1], dtype=np.float64).ravel()
    mdot0 = np.zeros(mesh.n_faces)
    mdot0[:mesh.n_interior] = np.asarray(fm["internal"][1], dtype=np.float64).ravel()
    for patch in mesh.patches:
        ent = fm["boundary"].get(patch.name)
        if ent and "value" in ent:
            mdot0[patch.start:patch.start + patch.n] = np.asarray(ent["value"][1], dtype=np.float64).ravel()
    return U0, p0, mdot0
