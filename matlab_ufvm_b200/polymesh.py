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
